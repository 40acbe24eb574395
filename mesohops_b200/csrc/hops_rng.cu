// Raw white noise of the FFT_FILTER model drawn on the device, the GPU
// replacement of noise/hops_noise.py:558-628 (_generate_noise_samples,
// _construct_indexing) and of the complex64 assembly at hops_noise.py:522-553.
//
// The reference gives L-operator l of a trajectory the stream
// PCG64(SEED).jumped(l) and draws 4(n_t-1) numbers from it with numpy's
// Generator.normal (SUM_GAUSSIAN) or Generator.random (BOX_MULLER).  Here one
// thread owns one (trajectory, L-operator) row and replays that stream:
//   * PCG64 is O'Neill's permuted congruential generator with 128-bit state,
//     multiplier 0x2360ed051fc65da44385df649fccf645, XSL-RR output taken after
//     the step; jumped(l) advances the state by l * 0x9e3779b97f4a7c15f39cc0605cedc835
//     steps (mod 2^128) with Brown's logarithmic-time LCG skip.  The caller
//     passes the un-jumped state and increment (numpy's PCG64(SEED).state), so
//     the seed hashing stays on the host.
//   * Uniform doubles are (raw >> 11) * 2^-53.
//   * Normals come from the 256-layer Marsaglia-Tsang ziggurat over a 52-bit
//     field (table and its derivation in hops_ziggurat_table.h and
//     make_ziggurat_table.py), with the exponential tail beyond r for layer 0.
//     Every product, sum and comparison is rounded as written (no fused
//     multiply-add), so the accept decisions and the returned doubles are those
//     of the same arithmetic on the host; only the rare tail draws (about 3e-4
//     of all draws) call log1p, whose last bit can differ between libraries.
//   * Draw d of a row lands in time slot s(d) (real part or Box-Muller radius
//     for d = 0, 2 mod 4; imaginary part or phase for d = 1, 3 mod 4) by the
//     closed form of _construct_indexing: d = 0, 1 -> slot 0; d = 4k-2, 4k-1 ->
//     slot k (k = 1 .. n_t-1); d = 4k, 4k+1 -> slot 2(n_t-1) - k (k = 1 .. n_t-2).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include "hops_ziggurat_table.h"

void hops_set_error_text(const char* msg);  // defined in hops_rk4.cu

namespace {

typedef unsigned __int128 u128;

constexpr u128 kPcgMult = ((u128)0x2360ed051fc65da4ull << 64) | 0x4385df649fccf645ull;
constexpr u128 kPcgJump = ((u128)0x9e3779b97f4a7c15ull << 64) | 0xf39cc0605cedc835ull;
constexpr double kZigR = 3.6541528853610088;
constexpr double kZigInvR = 1.0 / 3.6541528853610088;
constexpr double kTwoPi = 6.283185307179586;  // 2.0 * numpy.pi
constexpr uint64_t kMask52 = 0x000fffffffffffffull;

__constant__ double c_wi[256] = HOPS_ZIG_WI;
__constant__ unsigned long long c_ki[256] = HOPS_ZIG_KI;
__constant__ double c_fi[256] = HOPS_ZIG_FI;

struct ZigTable {
  double wi[256];
  double fi[256];
  unsigned long long ki[256];
};

struct Pcg {
  u128 s, inc;
};

__device__ __forceinline__ uint64_t pcg_next(Pcg& g) {
  g.s = g.s * kPcgMult + g.inc;
  const uint64_t x = (uint64_t)(g.s >> 64) ^ (uint64_t)g.s;
  const unsigned rot = (unsigned)(g.s >> 122);
  return (x >> rot) | (x << ((64u - rot) & 63u));
}

// State after `delta` steps: s_{n+delta} = A s_n + C with A = mult^delta and
// C = inc (mult^delta - 1) / (mult - 1), both built by squaring.
__device__ u128 pcg_advance(u128 s, u128 inc, u128 delta) {
  u128 acc_mult = 1, acc_plus = 0, cur_mult = kPcgMult, cur_plus = inc;
  while (delta) {
    if (delta & 1) {
      acc_mult *= cur_mult;
      acc_plus = acc_plus * cur_mult + cur_plus;
    }
    cur_plus = (cur_mult + 1) * cur_plus;
    cur_mult *= cur_mult;
    delta >>= 1;
  }
  return acc_mult * s + acc_plus;
}

__device__ __forceinline__ double next_double(Pcg& g) {
  return (double)(pcg_next(g) >> 11) * (1.0 / 9007199254740992.0);
}

__device__ double zig_normal(Pcg& g, const ZigTable& z) {
  for (;;) {
    uint64_t r = pcg_next(g);
    const int idx = (int)(r & 0xff);
    r >>= 8;
    const uint64_t field = (r >> 1) & kMask52;
    double x = __dmul_rn((double)field, z.wi[idx]);
    if (r & 1) x = -x;
    if (field < z.ki[idx]) return x;  // about 99 % of draws
    if (idx == 0) {
      for (;;) {
        const double xx = __dmul_rn(-kZigInvR, log1p(-next_double(g)));
        const double yy = -log1p(-next_double(g));
        if (__dadd_rn(yy, yy) > __dmul_rn(xx, xx))
          return ((field >> 8) & 1) ? -__dadd_rn(kZigR, xx) : __dadd_rn(kZigR, xx);
      }
    }
    const double height =
        __dadd_rn(__dmul_rn(__dadd_rn(z.fi[idx - 1], -z.fi[idx]), next_double(g)), z.fi[idx]);
    if (height < exp(__dmul_rn(__dmul_rn(-0.5, x), x))) return x;
  }
}

// Time slot of the draw pair starting at even draw d (see the header comment).
__device__ __forceinline__ long draw_slot(long d, long n1) {
  if (d == 0) return 0;
  if ((d & 3) == 2) return (d + 2) >> 2;
  return 2 * n1 - (d >> 2);
}

// rows = n_traj * n_lop; row = b * n_lop + j uses trajectory b's generator
// jumped lops[j] times and writes z[row][0 .. 2(n_t-1)).
__global__ void __launch_bounds__(128) k_raw_draws(const unsigned long long* __restrict__ states,
                                                   const int32_t* __restrict__ lops, int n_traj,
                                                   int n_lop, int n_t, int model,
                                                   float2* __restrict__ z) {
  __shared__ ZigTable tab;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    tab.wi[i] = c_wi[i];
    tab.fi[i] = c_fi[i];
    tab.ki[i] = c_ki[i];
  }
  __syncthreads();
  const long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= (long)n_traj * n_lop) return;
  const long b = row / n_lop;
  const int lop = lops[row - b * n_lop];
  const unsigned long long* st = states + 4 * b;
  Pcg g;
  g.inc = ((u128)st[2] << 64) | st[3];
  g.s = pcg_advance(((u128)st[0] << 64) | st[1], g.inc, (u128)(uint64_t)lop * kPcgJump);
  const long n1 = n_t - 1;
  float2* out = z + row * 2 * n1;
  for (long d = 0; d < 4 * n1; d += 2) {
    double a, c;
    if (model == 0) {
      a = zig_normal(g, tab);
      c = zig_normal(g, tab);
    } else {
      const double u = next_double(g);
      const double phi = next_double(g);
      const double rad = sqrt(__dmul_rn(-2.0, log(u)));
      double sn, cs;
      sincos(__dmul_rn(kTwoPi, phi), &sn, &cs);
      a = __dmul_rn(rad, cs);
      c = __dmul_rn(rad, sn);
    }
    out[draw_slot(d, n1)] = make_float2(__double2float_rn(a), __double2float_rn(c));
  }
}

thread_local char g_rerr[512];

int rerr(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_rerr, sizeof(g_rerr), fmt, ap);
  va_end(ap);
  hops_set_error_text(g_rerr);
  return code;
}

}  // namespace

extern "C" int hops_noise_draw(const uint64_t* seed_states_dev, int32_t n_traj,
                               const int32_t* lops_dev, int32_t n_lop, int32_t n_t,
                               int32_t model, float* z_dev, void* stream) {
  if (!seed_states_dev || !lops_dev || !z_dev || n_traj <= 0 || n_lop <= 0 || n_t < 2 ||
      (model != 0 && model != 1))
    return rerr(1, "hops_noise_draw: bad arguments (n_traj=%d n_lop=%d n_t=%d model=%d)", n_traj,
                n_lop, n_t, model);
  const long rows = (long)n_traj * n_lop;
  const int threads = 128;
  const long blocks = (rows + threads - 1) / threads;
  if (blocks > 0x7fffffffL) return rerr(1, "hops_noise_draw: %ld rows", rows);
  k_raw_draws<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
      reinterpret_cast<const unsigned long long*>(seed_states_dev), lops_dev, n_traj, n_lop, n_t,
      model, reinterpret_cast<float2*>(z_dev));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rerr(2, "hops_noise_draw: %s", cudaGetErrorString(e));
  return 0;
}
