// Raw white noise of the FFT_FILTER model drawn on the device, the GPU
// replacement of noise/hops_noise.py:558-628 (_generate_noise_samples,
// _construct_indexing) and of the complex64 assembly at hops_noise.py:522-553.
//
// The reference gives L-operator l of a trajectory the stream
// PCG64(SEED).jumped(l) and draws 4(n_t-1) numbers from it with numpy's
// Generator.normal (SUM_GAUSSIAN) or Generator.random (BOX_MULLER).  Here one
// warp owns one (trajectory, L-operator) row and replays that stream 32 words
// at a time: lane i holds word base + i (its own copy of the generator, moved
// 32 steps per batch by one affine map of the state), so the stream's serial
// recurrence is spread over the lanes.  A normal draw takes one word about
// 99 % of the time; the warp emits the run of such draws up to the first
// word that needs more (found by a ballot) in one store, then resolves that
// draw with the next words of the stream (shuffled from their lanes) exactly as
// the sequential sampler does:
//   * PCG64 is O'Neill's permuted congruential generator with 128-bit state,
//     multiplier 0x2360ed051fc65da44385df649fccf645, XSL-RR output taken after
//     the step; jumped(l) advances the state by l * 0x9e3779b97f4a7c15f39cc0605cedc835
//     steps (mod 2^128) with Brown's logarithmic-time LCG skip.  The caller
//     passes the un-jumped state and increment (numpy's PCG64(SEED).state),
//     which k_seed_states computes from integer SEEDs on the device.
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

#include "../../include/hops_b200.h"
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

// Affine map of `delta` steps: s -> mult * s + C with mult = mult^delta.
__device__ void pcg_skip(u128 inc, u128 delta, u128& mult, u128& plus) {
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
  mult = acc_mult;
  plus = acc_plus;
}

__device__ __forceinline__ uint64_t xsl_rr(u128 s) {
  const uint64_t x = (uint64_t)(s >> 64) ^ (uint64_t)s;
  const unsigned rot = (unsigned)(s >> 122);
  return (x >> rot) | (x << ((64u - rot) & 63u));
}

__device__ __forceinline__ double uniform53(uint64_t w) {
  return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

// Time slot of the draw pair starting at even draw d (see the header comment).
__device__ __forceinline__ long draw_slot(long d, long n1) {
  if (d == 0) return 0;
  if ((d & 3) == 2) return (d + 2) >> 2;
  return 2 * n1 - (d >> 2);
}

// The lanes' 32 consecutive words of one stream.
struct WarpStream {
  u128 t;        // this lane's state right after producing its word
  u128 a32, c32; // the 32-step map
  uint64_t w;    // this lane's word of the current batch
  __device__ __forceinline__ void next() {
    t = a32 * t + c32;
    w = xsl_rr(t);
  }
  __device__ __forceinline__ uint64_t word(int j) const { return __shfl_sync(0xffffffffu, w, j); }
};

// rows = n_traj * n_lop; warp `row` = b * n_lop + j uses trajectory b's
// generator jumped lops[j] times and writes the row's 4 (n_t - 1) draws as
// z[row][0 .. 2(n_t-1)) (complex64: real part of slot k at float 2k).
__global__ void __launch_bounds__(256) k_raw_draws(const unsigned long long* __restrict__ states,
                                                   const int32_t* __restrict__ lops, int n_traj,
                                                   int n_lop, int n_t, int model,
                                                   float* __restrict__ z) {
  __shared__ ZigTable tab;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    tab.wi[i] = c_wi[i];
    tab.fi[i] = c_fi[i];
    tab.ki[i] = c_ki[i];
  }
  __syncthreads();
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long row = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= (long)n_traj * n_lop) return;  // whole warps only
  const long b = row / n_lop;
  const int lop = lops[row - b * n_lop];
  const unsigned long long* st = states + 4 * b;
  const u128 inc = ((u128)st[2] << 64) | st[3];
  u128 m, c;
  // the row's stream: PCG64(SEED).jumped(lop); lane i starts at word i
  pcg_skip(inc, (u128)(uint64_t)lop * kPcgJump, m, c);
  const u128 s0 = m * (((u128)st[0] << 64) | st[1]) + c;
  WarpStream ws;
  pcg_skip(inc, (u128)(lane + 1), m, c);
  ws.t = m * s0 + c;
  ws.w = xsl_rr(ws.t);
  pcg_skip(inc, (u128)32, ws.a32, ws.c32);

  const long n1 = n_t - 1;
  const long total = 4 * n1;
  float* out = z + row * 4 * n1;
  if (model == 1) {
    // BOX_MULLER: one uniform per draw; the even lane of each pair writes the slot
    for (long base = 0; base < total; base += 32) {
      const double u = uniform53(ws.w);
      const double ph = __shfl_down_sync(FULL, u, 1);
      const long d = base + lane;
      if (!(lane & 1) && d < total) {
        const double rad = sqrt(__dmul_rn(-2.0, log(u)));
        double sn, cs;
        sincos(__dmul_rn(kTwoPi, ph), &sn, &cs);
        reinterpret_cast<float2*>(out)[draw_slot(d, n1)] =
            make_float2(__double2float_rn(__dmul_rn(rad, cs)), __double2float_rn(__dmul_rn(rad, sn)));
      }
      ws.next();
    }
    return;
  }
  auto put = [&](long d, double v) {
    out[2 * draw_slot(d & ~1L, n1) + (d & 1)] = __double2float_rn(v);
  };
  long done = 0;  // draws written
  int pos = 0;    // word of the batch where the next draw starts (warp-uniform)
  while (done < total) {
    const int idx = (int)(ws.w & 0xff);
    const uint64_t r8 = ws.w >> 8;
    const uint64_t field = (r8 >> 1) & kMask52;
    double x = __dmul_rn((double)field, tab.wi[idx]);
    if (r8 & 1) x = -x;
    const bool fast = field < tab.ki[idx];
    const unsigned slow = __ballot_sync(FULL, !fast) & (FULL << pos);
    const int k = slow ? __ffs(slow) - 1 : 32;
    if (lane >= pos && lane < k && done + (lane - pos) < total) put(done + (lane - pos), x);
    done += k - pos;
    if (k == 32) {
      ws.next();
      pos = 0;
      continue;
    }
    if (done >= total) break;
    // the draw starting at word k needs the words after it
    const int kidx = __shfl_sync(FULL, idx, k);
    const double kx = __shfl_sync(FULL, x, k);
    const uint64_t kfield = __shfl_sync(FULL, field, k);
    int j = k + 1;
    bool have = false;
    double v = 0.0;
    if (kidx != 0) {
      if (j == 32) {
        ws.next();
        j = 0;
      }
      const double u = uniform53(ws.word(j++));
      const double height =
          __dadd_rn(__dmul_rn(__dadd_rn(tab.fi[kidx - 1], -tab.fi[kidx]), u), tab.fi[kidx]);
      if (height < exp(__dmul_rn(__dmul_rn(-0.5, kx), kx))) {
        v = kx;
        have = true;
      }
    } else {
      // tail beyond r (Marsaglia): pairs of uniforms until one is accepted
      for (;;) {
        if (j == 32) {
          ws.next();
          j = 0;
        }
        const double u1 = uniform53(ws.word(j++));
        if (j == 32) {
          ws.next();
          j = 0;
        }
        const double u2 = uniform53(ws.word(j++));
        const double xx = __dmul_rn(-kZigInvR, log1p(-u1));
        const double yy = -log1p(-u2);
        if (__dadd_rn(yy, yy) > __dmul_rn(xx, xx)) {
          v = ((kfield >> 8) & 1) ? -__dadd_rn(kZigR, xx) : __dadd_rn(kZigR, xx);
          have = true;
          break;
        }
      }
    }
    if (have) {
      if (lane == 0) put(done, v);
      ++done;
    }
    if (j == 32) {
      ws.next();
      j = 0;
    }
    pos = j;
  }
}

// numpy's SeedSequence(SEED) for an integer SEED (O'Neill's seed_seq_fe
// hashing: a pool of four 32-bit words filled from the SEED's 32-bit words,
// least significant first, by a multiplicative hash; every pool word mixed
// into every other; the remaining SEED words mixed in; then generate_state(4,
// uint64) read from the pool with a second hash), followed by PCG64's seeding
// from those four words: increment = (w2:w3 << 1) | 1, state = step(step(0) +
// w0:w1).  One thread per trajectory; words[ptr[b] .. ptr[b+1]) is SEED b.
__global__ void k_seed_states(const uint32_t* __restrict__ words, const int32_t* __restrict__ ptr,
                              int n_traj, unsigned long long* __restrict__ states) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n_traj) return;
  const int w0 = ptr[b], nw = ptr[b + 1] - ptr[b];
  uint32_t hc = 0x43b0d7e5u;
  auto hashmix = [&](uint32_t v) {
    v ^= hc;
    hc *= 0x931e8875u;
    v *= hc;
    return v ^ (v >> 16);
  };
  auto mix = [](uint32_t x, uint32_t y) {
    uint32_t r = 0xca01f9ddu * x - 0x4973f715u * y;
    return r ^ (r >> 16);
  };
  uint32_t pool[4];
  for (int i = 0; i < 4; ++i) pool[i] = hashmix(i < nw ? words[w0 + i] : 0u);
  for (int src = 0; src < 4; ++src)
    for (int dst = 0; dst < 4; ++dst)
      if (src != dst) pool[dst] = mix(pool[dst], hashmix(pool[src]));
  for (int src = 4; src < nw; ++src)
    for (int dst = 0; dst < 4; ++dst) pool[dst] = mix(pool[dst], hashmix(words[w0 + src]));
  uint32_t hb = 0x8b51f9ddu, out[8];
  for (int i = 0; i < 8; ++i) {
    uint32_t v = pool[i & 3] ^ hb;
    hb *= 0x58f38dedu;
    v *= hb;
    out[i] = v ^ (v >> 16);
  }
  uint64_t v64[4];
  for (int i = 0; i < 4; ++i) v64[i] = (uint64_t)out[2 * i] | ((uint64_t)out[2 * i + 1] << 32);
  const u128 inc = ((((u128)v64[2] << 64) | v64[3]) << 1) | 1;
  u128 st = inc;                                   // step from state 0
  st += ((u128)v64[0] << 64) | v64[1];
  st = st * kPcgMult + inc;
  states[4 * b + 0] = (unsigned long long)(st >> 64);
  states[4 * b + 1] = (unsigned long long)st;
  states[4 * b + 2] = (unsigned long long)(inc >> 64);
  states[4 * b + 3] = (unsigned long long)inc;
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
    return rerr(HOPS_EINVAL, "hops_noise_draw: bad arguments (n_traj=%d n_lop=%d n_t=%d model=%d)",
                n_traj, n_lop, n_t, model);
  const long rows = (long)n_traj * n_lop;
  const int threads = 256;  // 8 rows (warps) per CTA
  const long blocks = (rows * 32 + threads - 1) / threads;
  if (blocks > 0x7fffffffL) return rerr(HOPS_EINVAL, "hops_noise_draw: %ld rows", rows);
  k_raw_draws<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
      reinterpret_cast<const unsigned long long*>(seed_states_dev), lops_dev, n_traj, n_lop, n_t,
      model, z_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rerr(HOPS_ECUDA, "hops_noise_draw: %s", cudaGetErrorString(e));
  return 0;
}

extern "C" int hops_noise_seed_states(const uint32_t* seed_words_dev, const int32_t* seed_ptr_dev,
                                      int32_t n_traj, uint64_t* seed_states_dev, void* stream) {
  if (!seed_words_dev || !seed_ptr_dev || !seed_states_dev || n_traj <= 0)
    return rerr(HOPS_EINVAL, "hops_noise_seed_states: bad arguments (n_traj=%d)", n_traj);
  k_seed_states<<<(n_traj + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      seed_words_dev, seed_ptr_dev, n_traj, reinterpret_cast<unsigned long long*>(seed_states_dev));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rerr(HOPS_ECUDA, "hops_noise_seed_states: %s", cudaGetErrorString(e));
  return 0;
}
