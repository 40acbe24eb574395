// RK4 propagation without any device allocation.
//
// Some callers cannot allocate device memory at the point where they step a
// trajectory: host codes that hand every byte of the GPU to their own memory
// pool (a cudaMalloc there fails or fragments the pool), and per-step plugin
// callbacks that must not synchronise the device (cudaMalloc / cudaFree may).
// hops_rk4_propagate_noalloc serves them: its stage vectors, accumulator and
// scalar workspace live in the fixed array below.
//
// The array is in a translation unit of its own, so it lives in its own CUDA
// module: under lazy module loading (the CUDA 12 default) a process pays its
// HOPS_NOALLOC_SCRATCH_BYTES on a GPU only once it has called this entry point
// there, and then keeps it until exit.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include "hops_common.cuh"

using namespace hops;

#define HOPS_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) unsigned char g_noalloc_scratch[HOPS_NOALLOC_SCRATCH_BYTES];

// Host code holds only a host-side stand-in for g_noalloc_scratch; the device
// address comes from cudaGetSymbolAddress with the device current.  It is
// cached per device together with the id of the CUDA context it was looked up
// in: after cudaDeviceReset (or any switch to another context) the module is
// loaded again, possibly at another address, and the lookup is repeated.
struct ScratchSlot {
  unsigned long long ctx_id;
  void* ptr;
};
static ScratchSlot g_slot[HOPS_NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

typedef CUresult (*PFN_ctxGetCurrent)(CUcontext*);
typedef CUresult (*PFN_ctxGetId)(CUcontext, unsigned long long*);

static int fail(int code, const char* fmt, const char* a) {
  char buf[384];
  snprintf(buf, sizeof(buf), fmt, a);
  hops_set_error_text(buf);
  return code;
}

// Id of the calling thread's current CUDA context (driver entry points looked
// up through the runtime, so the library needs no link against libcuda).
// Returns HOPS_OK, or -1 when the thread has no current context yet.
static int current_context_id(unsigned long long* id) {
  static PFN_ctxGetCurrent get_current = nullptr;
  static PFN_ctxGetId get_id = nullptr;
  if (!get_current || !get_id) {
    cudaDriverEntryPointQueryResult q1, q2;
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaError_t e1 = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000,
                                                      cudaEnableDefault, &q1);
    cudaError_t e2 = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000,
                                                      cudaEnableDefault, &q2);
    if (e1 != cudaSuccess || e2 != cudaSuccess || !f1 || !f2 ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess)
      return fail(HOPS_ECUDA, "no-allocation propagate: driver entry points unavailable (%s)",
                  cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    get_current = reinterpret_cast<PFN_ctxGetCurrent>(f1);
    get_id = reinterpret_cast<PFN_ctxGetId>(f2);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS)
    return fail(HOPS_ECUDA, "no-allocation propagate: %s", "cuCtxGetCurrent failed");
  if (!ctx) return -1;
  if (get_id(ctx, id) != CUDA_SUCCESS)
    return fail(HOPS_ECUDA, "no-allocation propagate: %s", "cuCtxGetId failed");
  return HOPS_OK;
}

static int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(HOPS_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= HOPS_NOALLOC_MAX_DEVICES)
    return fail(HOPS_ENOTSUP, "no-allocation propagate: %s",
                "device index beyond its 64-entry table");
  unsigned long long ctx = 0;
  int rc = current_context_id(&ctx);
  if (rc > 0) return rc;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (rc < 0 || !g_slot[dev].ptr || g_slot[dev].ctx_id != ctx) {
    void* p = nullptr;
    // also makes the device's primary context current when the thread had none
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(HOPS_ECUDA, "cudaGetSymbolAddress(no-allocation scratch): %s",
                  cudaGetErrorString(e));
    if ((rc = current_context_id(&ctx)))
      return rc > 0 ? rc : fail(HOPS_ECUDA, "no-allocation propagate: %s", "no CUDA context");
    g_slot[dev].ptr = p;
    g_slot[dev].ctx_id = ctx;
  }
  *out = g_slot[dev].ptr;
  return HOPS_OK;
}

// Left-over contents of the shared array are made harmless: every
// trajectory's pending scale (both copies of it) is reset to 1, and in the
// mixed mode the complex64 copy of phi that the first stage reads is rebuilt.
// Everything else in the array is written before it is read.
template <typename PT, typename ST>
__global__ void k_noalloc_prep(double* ws, int stride, size_t scale_off, int B, const PT* phi,
                               ST* shadow, size_t E) {
  const size_t i0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t n = (size_t)gridDim.x * blockDim.x;
  for (size_t b = i0; b < (size_t)B; b += n) {
    ws[b * stride] = 1.0;
    ws[scale_off + b] = 1.0;
  }
  if (shadow)
    for (size_t e = i0; e < E; e += n) {
      const PT v = phi[e];
      shadow[e] = ST{(float)v.x, (float)v.y};
    }
}

extern "C" size_t hops_noalloc_scratch_bytes(const hops_structure* st, int32_t n_traj,
                                             int32_t precision) {
  if (!st || n_traj <= 0 || st->n_hier <= 0 || st->n_state <= 0) return 0;
  const size_t E = (size_t)st->n_hier * st->n_state * n_traj;
  const size_t sv = precision == HOPS_PREC_C128 ? 16 : 8;
  size_t bytes = 3 * E * sv;                          // acc, y0, y1
  if (precision == HOPS_PREC_MIXED) bytes += E * sv;  // complex64 copy of phi
  bytes = (bytes + 255) & ~(size_t)255;
  bytes += BatchLayout(st->n_state, st->n_mode, st->n_lop, n_traj).total * sizeof(double);
  return bytes;
}

extern "C" int hops_rk4_propagate_noalloc(const hops_structure* st, int32_t n_traj,
                                          int32_t precision, int32_t eom, void* phi_dev,
                                          double* zmem_dev, const float* noise1_dev,
                                          int32_t n_t1, const float* noise2_dev, int32_t n_t2,
                                          int32_t it0, int32_t di, int32_t n_steps,
                                          double tau_over_hbar, double* psi_out_dev,
                                          int32_t* status_dev, void* stream) {
  if (!st || n_traj <= 0 || !phi_dev || !zmem_dev || !status_dev) {
    hops_set_error_text("no-allocation propagate: bad arguments");
    return HOPS_EINVAL;
  }
  const size_t need = hops_noalloc_scratch_bytes(st, n_traj, precision);
  if (need > (size_t)HOPS_NOALLOC_SCRATCH_BYTES) {
    char buf[384];
    snprintf(buf, sizeof(buf),
             "no-allocation propagate needs %zu bytes of scratch, more than its %u-byte static "
             "area; use hops_rk4_propagate with caller-allocated buffers",
             need, (unsigned)HOPS_NOALLOC_SCRATCH_BYTES);
    hops_set_error_text(buf);
    return HOPS_EINVAL;
  }
  // The batch is laid over the array by offsets alone, so every argument check
  // runs (on a placeholder base) before the array is looked up or anything is
  // launched: a rejected call leaves the device and the status words untouched.
  const size_t E = (size_t)st->n_hier * st->n_state * n_traj;
  const size_t sv = precision == HOPS_PREC_C128 ? 16 : 8;
  auto lay_out = [&](unsigned char* p, hops_batch* bt) {
    memset(bt, 0, sizeof(*bt));
    bt->n_traj = n_traj;
    bt->precision = precision;
    bt->eom = eom;
    bt->phi = phi_dev;
    bt->acc = p;
    bt->y0 = p + E * sv;
    bt->y1 = p + 2 * E * sv;
    size_t off = 3 * E * sv;
    if (precision == HOPS_PREC_MIXED) {
      bt->phi_lo = p + off;
      off += E * sv;
    }
    off = (off + 255) & ~(size_t)255;
    bt->work = reinterpret_cast<double*>(p + off);
    bt->zmem = zmem_dev;
    bt->noise1 = noise1_dev;
    bt->n_t1 = n_t1;
    bt->noise2 = noise2_dev;
    bt->n_t2 = n_t2;
    bt->status = status_dev;
  };
  hops_batch bt;
  lay_out(reinterpret_cast<unsigned char*>((uintptr_t)256), &bt);
  int rc = hops_check_propagate_args(st, &bt, it0, di, n_steps);
  if (rc) return rc;
  void* base = nullptr;
  if ((rc = noalloc_scratch(&base))) return rc;
  lay_out(static_cast<unsigned char*>(base), &bt);
  cudaStream_t s = (cudaStream_t)stream;
  const ScalarLayout lay(st->n_state, st->n_mode, st->n_lop);
  const BatchLayout bl(st->n_state, st->n_mode, st->n_lop, n_traj);
  const size_t work = precision == HOPS_PREC_MIXED ? E : (size_t)n_traj;
  int blocks = (int)std::min<size_t>((work + 255) / 256, (size_t)148 * 8);
  if (blocks < 1) blocks = 1;
  if (precision == HOPS_PREC_MIXED)
    k_noalloc_prep<double2, float2><<<blocks, 256, 0, s>>>(
        bt.work, lay.stride, bl.scaleB, n_traj, (const double2*)phi_dev, (float2*)bt.phi_lo, E);
  else
    k_noalloc_prep<double2, float2><<<blocks, 256, 0, s>>>(bt.work, lay.stride, bl.scaleB,
                                                           n_traj, nullptr, nullptr, 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(HOPS_ECUDA, "no-allocation prep launch: %s", cudaGetErrorString(e));
  return hops_rk4_propagate(st, &bt, it0, di, n_steps, tau_over_hbar, psi_out_dev, stream);
}
