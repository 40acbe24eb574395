// Host-array entry points: a caller with plain host arrays (any language with a
// C FFI) builds a structure and a batch whose device memory the library owns,
// sets states and noise from host buffers and reads psi(t) and the state back
// into host buffers.  The derived tables (f32 copies, L^H, the site-projector
// form, first-level aux, K2_k) are computed here from the minimal description,
// exactly as the package's Python table builder does.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <complex>
#include <vector>
#include "hops_common.cuh"

using namespace hops;

namespace {

using cd = std::complex<double>;

int fail(int code, const char* fmt, ...) {
  char buf[384];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  hops_set_error_text(buf);
  return code;
}

#define HOST_CUDA(expr)                                                               \
  do {                                                                                \
    cudaError_t e_ = (expr);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(HOPS_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                  __LINE__);                                                          \
  } while (0)

// a / b by Smith's method with a reciprocal (R. L. Smith, "Algorithm 116:
// Complex division", CACM 5(8), 1962), the form numpy evaluates, so the
// quotient g/w is bit-identical to the Python table builder's.
cd cdiv(cd a, cd b) {
  const double br = b.real(), bi = b.imag();
  if (fabs(br) >= fabs(bi)) {
    const double rat = bi / br;
    const double scl = 1.0 / (br + bi * rat);
    return cd((a.real() + a.imag() * rat) * scl, (a.imag() - a.real() * rat) * scl);
  }
  const double rat = br / bi;
  const double scl = 1.0 / (bi + br * rat);
  return cd((a.real() * rat + a.imag()) * scl, (a.imag() * rat - a.real()) * scl);
}

// (ar + i ai)(br + i bi) with the textbook formula, as numpy evaluates it
cd cmul_h(cd a, cd b) {
  return cd(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

cd ld(const double* p, size_t i) { return cd(p[2 * i], p[2 * i + 1]); }

// Packed host image of every table, uploaded with one copy.
struct Packer {
  std::vector<unsigned char> buf;
  size_t put(const void* src, size_t bytes) {
    const size_t off = (buf.size() + 255) & ~(size_t)255;
    buf.resize(off + std::max<size_t>(bytes, 16), 0);
    if (bytes && src) memcpy(buf.data() + off, src, bytes);   // src NULL: reserve only
    return off;
  }
  size_t cplx(const std::vector<cd>& v) {
    std::vector<double> d(2 * v.size());
    for (size_t i = 0; i < v.size(); ++i) {
      d[2 * i] = v[i].real();
      d[2 * i + 1] = v[i].imag();
    }
    return put(d.data(), d.size() * sizeof(double));
  }
  size_t cplx_f(const std::vector<cd>& v) {
    std::vector<float> d(2 * v.size());
    for (size_t i = 0; i < v.size(); ++i) {
      d[2 * i] = (float)v[i].real();
      d[2 * i + 1] = (float)v[i].imag();
    }
    return put(d.data(), d.size() * sizeof(float));
  }
  size_t i32(const std::vector<int32_t>& v) { return put(v.data(), v.size() * sizeof(int32_t)); }
};

// CSR (row-major entry order) of n_mat dense n x n matrices, block j at
// ptr[j*(n+1) ...] with absolute offsets.
void csr_of_dense(const std::vector<std::vector<cd>>& mats, int n, std::vector<int32_t>& ptr,
                  std::vector<int32_t>& col, std::vector<cd>& val) {
  ptr.assign(mats.size() * (n + 1), 0);
  col.clear();
  val.clear();
  for (size_t j = 0; j < mats.size(); ++j) {
    for (int r = 0; r < n; ++r) {
      ptr[j * (n + 1) + r] = (int32_t)col.size();
      for (int c = 0; c < n; ++c) {
        const cd v = mats[j][(size_t)r * n + c];
        if (v != cd(0.0, 0.0)) {
          col.push_back(c);
          val.push_back(v);
        }
      }
    }
    ptr[j * (n + 1) + n] = (int32_t)col.size();
  }
}

}  // namespace

struct hops_structure_owned {
  hops_structure host;       // device pointers, host memory
  hops_structure* dev;       // device copy of `host`
  void* buffer;              // every table
};

extern "C" int hops_structure_upload(const hops_structure_desc* d, void* stream,
                                     hops_structure_owned** out) {
  if (!d || !out) return fail(HOPS_EINVAL, "hops_structure_upload: null argument");
  *out = nullptr;
  const int N = d->n_hier, S = d->n_state, M = d->n_mode, L = d->n_lop;
  if (N <= 0 || S <= 0 || M < 0 || L < 0 || (long)N * S >= (1L << 31))
    return fail(HOPS_EINVAL, "hops_structure_upload: bad sizes n_hier=%d n_state=%d n_mode=%d "
                "n_lop=%d", N, S, M, L);
  if (!d->up_ptr || !d->dn_ptr || !d->hamiltonian || (M > 0 && (!d->mode_lop || !d->mode_g ||
      !d->mode_w)) || (L > 0 && !d->lops))
    return fail(HOPS_EINVAL, "hops_structure_upload: null table");
  const int n_up = d->up_ptr[N], n_dn = d->dn_ptr[N];
  if (d->up_ptr[0] != 0 || d->dn_ptr[0] != 0 || n_up < 0 || n_dn < 0 ||
      (n_up > 0 && (!d->up_aux || !d->up_mode)) ||
      (n_dn > 0 && (!d->dn_aux || !d->dn_mode || !d->dn_k)))
    return fail(HOPS_EINVAL, "hops_structure_upload: bad connection lists");
  for (int a = 0; a < N; ++a)
    if (d->up_ptr[a + 1] < d->up_ptr[a] || d->dn_ptr[a + 1] < d->dn_ptr[a])
      return fail(HOPS_EINVAL, "hops_structure_upload: connection pointers decrease at aux %d", a);
  for (int p = 0; p < n_up; ++p)
    if (d->up_aux[p] < 0 || d->up_aux[p] >= N || d->up_mode[p] < 0 || d->up_mode[p] >= M)
      return fail(HOPS_EINVAL, "hops_structure_upload: up connection %d out of range", p);
  for (int p = 0; p < n_dn; ++p)
    if (d->dn_aux[p] < 0 || d->dn_aux[p] >= N || d->dn_mode[p] < 0 || d->dn_mode[p] >= M ||
        d->dn_k[p] < 1)
      return fail(HOPS_EINVAL, "hops_structure_upload: down connection %d out of range", p);
  for (int m = 0; m < M; ++m) {
    if (d->mode_lop[m] < 0 || d->mode_lop[m] >= L)
      return fail(HOPS_EINVAL, "hops_structure_upload: mode %d has L index %d of %d", m,
                  d->mode_lop[m], L);
    if (d->mode_w[2 * m] == 0.0 && d->mode_w[2 * m + 1] == 0.0)
      return fail(HOPS_EINVAL, "hops_structure_upload: mode %d has w = 0", m);
  }
  if (N > 0 && d->dn_ptr[1] != 0)
    return fail(HOPS_EINVAL, "hops_structure_upload: aux 0 must be the physical wavefunction");

  // ---- state / mode tables
  std::vector<std::vector<cd>> lops(L, std::vector<cd>((size_t)S * S));
  std::vector<int32_t> lop_active(L, 0), lop_site(L, 0);
  std::vector<cd> lop_sval(L, cd(0.0, 0.0));
  bool is_site = true;
  for (int j = 0; j < L; ++j) {
    int nnz = 0, r0 = -1, c0 = -1;
    for (int r = 0; r < S; ++r)
      for (int c = 0; c < S; ++c) {
        const cd v = ld(d->lops, ((size_t)j * S + r) * S + c);
        lops[j][(size_t)r * S + c] = v;
        if (v != cd(0.0, 0.0)) {
          ++nnz;
          r0 = r;
          c0 = c;
        }
      }
    lop_active[j] = nnz > 0;
    if (nnz == 1 && r0 == c0) {
      lop_site[j] = r0;
      lop_sval[j] = lops[j][(size_t)r0 * S + c0];
    } else if (nnz == 0) {
      lop_site[j] = -1;
    } else {
      is_site = false;
    }
  }
  std::vector<std::vector<cd>> lh(L, std::vector<cd>((size_t)S * S));
  for (int j = 0; j < L; ++j)
    for (int r = 0; r < S; ++r)
      for (int c = 0; c < S; ++c) lh[j][(size_t)r * S + c] = std::conj(lops[j][(size_t)c * S + r]);
  std::vector<int32_t> l_ptr, l_col, lh_ptr, lh_col;
  std::vector<cd> l_val, lh_val;
  csr_of_dense(lops, S, l_ptr, l_col, l_val);
  csr_of_dense(lh, S, lh_ptr, lh_col, lh_val);
  // -i H; for site projectors the diagonal joins the per-state coefficient
  std::vector<std::vector<cd>> mh(1, std::vector<cd>((size_t)S * S));
  std::vector<cd> h_diag;
  for (int r = 0; r < S; ++r)
    for (int c = 0; c < S; ++c) {
      const cd h = ld(d->hamiltonian, (size_t)r * S + c);
      const cd v(h.imag(), -h.real());
      if (is_site && r == c) h_diag.push_back(v);
      else mh[0][(size_t)r * S + c] = v;
    }
  std::vector<int32_t> h_ptr, h_col;
  std::vector<cd> h_val;
  csr_of_dense(mh, S, h_ptr, h_col, h_val);
  std::vector<cd> G(M), W(M), GW(M), GWV(M);
  std::vector<int32_t> mode_lop(M), mode_site(M);
  for (int m = 0; m < M; ++m) {
    G[m] = ld(d->mode_g, m);
    W[m] = ld(d->mode_w, m);
    GW[m] = cdiv(G[m], W[m]);
    mode_lop[m] = d->mode_lop[m];
    mode_site[m] = lop_site[mode_lop[m]];
    GWV[m] = cmul_h(GW[m], lop_sval[mode_lop[m]]);
  }
  bool has_lt = false;
  std::vector<cd> lt(L, cd(0.0, 0.0));
  if (d->lt_coef)
    for (int j = 0; j < L; ++j) {
      lt[j] = ld(d->lt_coef, j);
      has_lt |= lt[j] != cd(0.0, 0.0);
    }
  std::vector<int32_t> l2_ptr, l2_col;
  std::vector<cd> l2_val;
  if (has_lt) {
    std::vector<std::vector<cd>> l2(L, std::vector<cd>((size_t)S * S, cd(0.0, 0.0)));
    for (int j = 0; j < L; ++j)
      for (int r = 0; r < S; ++r)
        for (int c = 0; c < S; ++c) {
          cd acc(0.0, 0.0);
          for (int k = 0; k < S; ++k)
            acc += cmul_h(lops[j][(size_t)r * S + k], lops[j][(size_t)k * S + c]);
          l2[j][(size_t)r * S + c] = acc;
        }
    csr_of_dense(l2, S, l2_ptr, l2_col, l2_val);
  }

  // ---- aux tables
  std::vector<cd> k_decay(N, cd(0.0, 0.0)), dn_coef(n_dn), dn_coef_site(n_dn);
  std::vector<int32_t> up_site(n_up), dn_site(n_dn), first_of_mode(M, -1);
  int max_up = 0, max_dn = 0, n_up_prefix = 0;
  for (int a = 0; a < N; ++a) {
    max_up = std::max(max_up, d->up_ptr[a + 1] - d->up_ptr[a]);
    if (d->up_ptr[a + 1] > d->up_ptr[a]) n_up_prefix = a + 1;
    max_dn = std::max(max_dn, d->dn_ptr[a + 1] - d->dn_ptr[a]);
    cd s(0.0, 0.0);
    for (int p = d->dn_ptr[a]; p < d->dn_ptr[a + 1]; ++p) s += (double)d->dn_k[p] * W[d->dn_mode[p]];
    k_decay[a] = -s;
    if (d->dn_ptr[a + 1] - d->dn_ptr[a] == 1) {
      const int p = d->dn_ptr[a];
      if (d->dn_k[p] == 1 && d->dn_aux[p] == 0) first_of_mode[d->dn_mode[p]] = a;
    }
  }
  for (int p = 0; p < n_dn; ++p) {
    const int m = d->dn_mode[p];
    dn_coef[p] = (double)d->dn_k[p] * W[m];
    dn_coef_site[p] = cmul_h(dn_coef[p], std::conj(lop_sval[mode_lop[m]]));
    dn_site[p] = mode_site[m];
  }
  for (int p = 0; p < n_up; ++p) up_site[p] = mode_site[d->up_mode[p]];
  std::vector<int32_t> first_aux, first_mode;
  for (int m = 0; m < M; ++m)
    if (first_of_mode[m] >= 0) {
      first_aux.push_back(first_of_mode[m]);
      first_mode.push_back(m);
    }

  // ---- pack and upload
  Packer pk;
  std::vector<int32_t> up_ptr(d->up_ptr, d->up_ptr + N + 1), dn_ptr(d->dn_ptr, d->dn_ptr + N + 1);
  std::vector<int32_t> up_aux(d->up_aux, d->up_aux + n_up), up_mode(d->up_mode, d->up_mode + n_up);
  std::vector<int32_t> dn_aux(d->dn_aux, d->dn_aux + n_dn), dn_mode(d->dn_mode, d->dn_mode + n_dn);
  const size_t o_kd = pk.cplx(k_decay), o_kdf = pk.cplx_f(k_decay);
  const size_t o_upp = pk.i32(up_ptr), o_upa = pk.i32(up_aux), o_upm = pk.i32(up_mode);
  const size_t o_dnp = pk.i32(dn_ptr), o_dna = pk.i32(dn_aux), o_dnm = pk.i32(dn_mode);
  const size_t o_dnc = pk.cplx(dn_coef), o_dncf = pk.cplx_f(dn_coef);
  const size_t o_ml = pk.i32(mode_lop), o_mg = pk.cplx(G), o_mw = pk.cplx(W);
  const size_t o_mgw = pk.cplx(GW), o_mgwf = pk.cplx_f(GW);
  const size_t o_fa = pk.i32(first_aux), o_fm = pk.i32(first_mode);
  const size_t o_lp = pk.i32(l_ptr), o_lc = pk.i32(l_col), o_lv = pk.cplx(l_val), o_lvf = pk.cplx_f(l_val);
  const size_t o_hp_ = pk.i32(lh_ptr), o_hc_ = pk.i32(lh_col), o_hv_ = pk.cplx(lh_val),
               o_hvf_ = pk.cplx_f(lh_val);
  const size_t o_la = pk.i32(lop_active), o_ls = pk.i32(lop_site), o_lsv = pk.cplx(lop_sval);
  const size_t o_hp = pk.i32(h_ptr), o_hc = pk.i32(h_col), o_hv = pk.cplx(h_val), o_hvf = pk.cplx_f(h_val);
  const size_t o_ms = pk.i32(mode_site), o_gwv = pk.cplx(GWV), o_gwvf = pk.cplx_f(GWV);
  const size_t o_dcs = pk.cplx(dn_coef_site), o_dcsf = pk.cplx_f(dn_coef_site);
  const size_t o_us = pk.i32(up_site), o_ds = pk.i32(dn_site);
  const size_t o_hd = is_site ? pk.cplx(h_diag) : 0;
  size_t o_lt = 0, o_l2p = 0, o_l2c = 0, o_l2v = 0;
  if (has_lt) {
    o_lt = pk.cplx(lt);
    o_l2p = pk.i32(l2_ptr);
    o_l2c = pk.i32(l2_col);
    o_l2v = pk.cplx(l2_val);
  }
  const size_t o_struct = pk.put(nullptr, sizeof(hops_structure));

  hops_structure_owned* own = (hops_structure_owned*)calloc(1, sizeof(hops_structure_owned));
  if (!own) return fail(HOPS_EINVAL, "hops_structure_upload: out of host memory");
  cudaError_t e = cudaMalloc(&own->buffer, pk.buf.size());
  if (e != cudaSuccess) {
    free(own);
    return fail(HOPS_ECUDA, "hops_structure_upload: cudaMalloc of %zu bytes: %s", pk.buf.size(),
                cudaGetErrorString(e));
  }
  unsigned char* base = static_cast<unsigned char*>(own->buffer);
  hops_structure& st = own->host;
  memset(&st, 0, sizeof(st));
  st.n_hier = N;
  st.n_state = S;
  st.n_mode = M;
  st.n_lop = L;
  st.n_first = (int32_t)first_aux.size();
  st.n_up = n_up;
  st.n_dn = n_dn;
  st.site_projector = is_site ? 1 : 0;
  st.max_up = max_up;
  st.max_dn = max_dn;
  st.n_up_prefix = n_up_prefix;
#define AT(T, o) reinterpret_cast<T>(base + (o))
  st.k_decay = AT(const double*, o_kd);
  st.k_decay_f = AT(const float*, o_kdf);
  st.up_ptr = AT(const int32_t*, o_upp);
  st.up_aux = AT(const int32_t*, o_upa);
  st.up_mode = AT(const int32_t*, o_upm);
  st.dn_ptr = AT(const int32_t*, o_dnp);
  st.dn_aux = AT(const int32_t*, o_dna);
  st.dn_mode = AT(const int32_t*, o_dnm);
  st.dn_coef = AT(const double*, o_dnc);
  st.dn_coef_f = AT(const float*, o_dncf);
  st.mode_lop = AT(const int32_t*, o_ml);
  st.mode_g = AT(const double*, o_mg);
  st.mode_w = AT(const double*, o_mw);
  st.mode_gw = AT(const double*, o_mgw);
  st.mode_gw_f = AT(const float*, o_mgwf);
  st.first_aux = AT(const int32_t*, o_fa);
  st.first_mode = AT(const int32_t*, o_fm);
  st.l_ptr = AT(const int32_t*, o_lp);
  st.l_col = AT(const int32_t*, o_lc);
  st.l_val = AT(const double*, o_lv);
  st.l_val_f = AT(const float*, o_lvf);
  st.lh_ptr = AT(const int32_t*, o_hp_);
  st.lh_col = AT(const int32_t*, o_hc_);
  st.lh_val = AT(const double*, o_hv_);
  st.lh_val_f = AT(const float*, o_hvf_);
  st.lop_active = AT(const int32_t*, o_la);
  st.lop_site = AT(const int32_t*, o_ls);
  st.lop_sval = AT(const double*, o_lsv);
  st.h_ptr = AT(const int32_t*, o_hp);
  st.h_col = AT(const int32_t*, o_hc);
  st.h_val = AT(const double*, o_hv);
  st.h_val_f = AT(const float*, o_hvf);
  st.mode_site = AT(const int32_t*, o_ms);
  st.mode_gwv = AT(const double*, o_gwv);
  st.mode_gwv_f = AT(const float*, o_gwvf);
  st.dn_coef_site = AT(const double*, o_dcs);
  st.dn_coef_site_f = AT(const float*, o_dcsf);
  st.up_site = AT(const int32_t*, o_us);
  st.dn_site = AT(const int32_t*, o_ds);
  st.h_diag = is_site ? AT(const double*, o_hd) : nullptr;
  if (has_lt) {
    st.lt_coef = AT(const double*, o_lt);
    st.l2_ptr = AT(const int32_t*, o_l2p);
    st.l2_col = AT(const int32_t*, o_l2c);
    st.l2_val = AT(const double*, o_l2v);
  }
  own->dev = AT(hops_structure*, o_struct);
#undef AT
  memcpy(pk.buf.data() + o_struct, &st, sizeof(st));
  cudaStream_t s = (cudaStream_t)stream;
  e = cudaMemcpyAsync(own->buffer, pk.buf.data(), pk.buf.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // the host image is freed on return
  if (e != cudaSuccess) {
    cudaFree(own->buffer);
    free(own);
    return fail(HOPS_ECUDA, "hops_structure_upload: copy: %s", cudaGetErrorString(e));
  }
  *out = own;
  return HOPS_OK;
}

extern "C" const hops_structure* hops_structure_host_view(const hops_structure_owned* s) {
  return s ? &s->host : nullptr;
}

extern "C" const hops_structure* hops_structure_device_view(const hops_structure_owned* s) {
  return s ? s->dev : nullptr;
}

extern "C" int hops_structure_destroy(hops_structure_owned* s) {
  if (!s) return HOPS_OK;
  cudaError_t e = cudaFree(s->buffer);
  free(s);
  if (e != cudaSuccess) return fail(HOPS_ECUDA, "hops_structure_destroy: %s", cudaGetErrorString(e));
  return HOPS_OK;
}

// ------------------------------------------------------------------ batches --
namespace {
struct OwnedBatch {
  hops_batch bt;          // first member: a hops_batch* of this batch is an OwnedBatch*
  void* vectors;          // phi, acc | y0 | y1 (contiguous), phi_lo
  void* small;            // zmem, work, status
  void* noise;            // noise1 | noise2
  size_t noise_bytes;
  double* psi;            // [cap] complex128 staging of psi(t)
  size_t psi_cap;         // complex elements
  int32_t n_hier, n_state, n_mode, n_lop;
};

size_t elem_bytes(int prec) { return prec == HOPS_PREC_C128 ? 16 : 8; }
size_t state_bytes(int prec) { return prec == HOPS_PREC_C64 ? 8 : 16; }

template <typename PT>
__global__ void k_state_in(const double2* in, PT* phi, float2* phi_lo, int B, size_t NS) {
  const size_t E = NS * B;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < E;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t as = e / B, b = e - as * B;
    const double2 v = in[b * NS + as];
    if constexpr (sizeof(PT) == 16) phi[e] = v;
    else phi[e] = make_float2((float)v.x, (float)v.y);
    if (phi_lo) phi_lo[e] = make_float2((float)v.x, (float)v.y);
  }
}

template <typename PT>
__global__ void k_state_out(const PT* phi, double2* out, int B, size_t NS) {
  const size_t E = NS * B;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < E;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t b = e / NS, as = e - b * NS;
    const PT v = phi[as * B + b];
    out[e] = make_double2((double)v.x, (double)v.y);
  }
}

int grid_of(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }
}  // namespace

extern "C" int hops_batch_create(const hops_structure* st, int32_t n_traj, int32_t precision,
                                 int32_t eom, hops_batch** out) {
  if (!st || !out || n_traj <= 0) return fail(HOPS_EINVAL, "hops_batch_create: bad arguments");
  *out = nullptr;
  if (precision != HOPS_PREC_C128 && precision != HOPS_PREC_C64 && precision != HOPS_PREC_MIXED)
    return fail(HOPS_EINVAL, "hops_batch_create: unknown precision %d", precision);
  if (eom < 0 || eom > 2) return fail(HOPS_EINVAL, "hops_batch_create: unknown eom %d", eom);
  OwnedBatch* ob = (OwnedBatch*)calloc(1, sizeof(OwnedBatch));
  if (!ob) return fail(HOPS_EINVAL, "hops_batch_create: out of host memory");
  ob->n_hier = st->n_hier;
  ob->n_state = st->n_state;
  ob->n_mode = st->n_mode;
  ob->n_lop = st->n_lop;
  const size_t E = (size_t)st->n_hier * st->n_state * n_traj;
  const size_t sv = elem_bytes(precision), sp = state_bytes(precision);
  const size_t phi_b = (E * sp + 255) & ~(size_t)255;
  const size_t stage_b = (3 * E * sv + 255) & ~(size_t)255;
  const size_t lo_b = precision == HOPS_PREC_MIXED ? E * 8 : 0;
  const size_t zm_b = ((size_t)n_traj * std::max(st->n_mode, 1) * 16 + 255) & ~(size_t)255;
  const size_t ws_b = (BatchLayout(st->n_state, st->n_mode, st->n_lop, n_traj).total * 8 + 255) &
                      ~(size_t)255;
  const size_t stat_b = (size_t)n_traj * 4;
  cudaError_t e = cudaMalloc(&ob->vectors, phi_b + stage_b + lo_b);
  if (e == cudaSuccess) e = cudaMalloc(&ob->small, zm_b + ws_b + stat_b);
  if (e != cudaSuccess) {
    cudaFree(ob->vectors);
    free(ob);
    return fail(HOPS_ECUDA, "hops_batch_create: cudaMalloc: %s", cudaGetErrorString(e));
  }
  unsigned char* v = static_cast<unsigned char*>(ob->vectors);
  unsigned char* sm = static_cast<unsigned char*>(ob->small);
  hops_batch& bt = ob->bt;
  bt.n_traj = n_traj;
  bt.precision = precision;
  bt.eom = eom;
  bt.phi = v;
  bt.acc = v + phi_b;
  bt.y0 = v + phi_b + E * sv;
  bt.y1 = v + phi_b + 2 * E * sv;
  bt.phi_lo = lo_b ? v + phi_b + stage_b : nullptr;
  bt.zmem = reinterpret_cast<double*>(sm);
  bt.work = reinterpret_cast<double*>(sm + zm_b);
  bt.status = reinterpret_cast<int32_t*>(sm + zm_b + ws_b);
  e = cudaMemset(ob->vectors, 0, phi_b + stage_b + lo_b);
  if (e == cudaSuccess) e = cudaMemset(ob->small, 0, zm_b + ws_b + stat_b);
  if (e != cudaSuccess) {
    cudaFree(ob->vectors);
    cudaFree(ob->small);
    free(ob);
    return fail(HOPS_ECUDA, "hops_batch_create: cudaMemset: %s", cudaGetErrorString(e));
  }
  int rc = hops_batch_reset(st, &bt, nullptr);
  if (rc == HOPS_OK && (e = cudaStreamSynchronize(nullptr)) != cudaSuccess)
    rc = fail(HOPS_ECUDA, "hops_batch_create: %s", cudaGetErrorString(e));
  if (rc) {
    cudaFree(ob->vectors);
    cudaFree(ob->small);
    free(ob);
    return rc;
  }
  *out = &ob->bt;
  return HOPS_OK;
}

extern "C" int hops_batch_destroy(hops_batch* bt) {
  if (!bt) return HOPS_OK;
  OwnedBatch* ob = reinterpret_cast<OwnedBatch*>(bt);
  cudaError_t e1 = cudaFree(ob->vectors), e2 = cudaFree(ob->small);
  cudaError_t e3 = cudaFree(ob->noise), e4 = cudaFree(ob->psi);
  free(ob);
  for (cudaError_t e : {e1, e2, e3, e4})
    if (e != cudaSuccess) return fail(HOPS_ECUDA, "hops_batch_destroy: %s", cudaGetErrorString(e));
  return HOPS_OK;
}

extern "C" int hops_batch_set_state_host(const hops_structure* st, hops_batch* bt,
                                         const double* phi_host, const double* zmem_host,
                                         void* stream) {
  if (!st || !bt || !phi_host) return fail(HOPS_EINVAL, "hops_batch_set_state_host: null argument");
  OwnedBatch* ob = reinterpret_cast<OwnedBatch*>(bt);
  if (ob->n_hier != st->n_hier || ob->n_state != st->n_state)
    return fail(HOPS_EINVAL, "hops_batch_set_state_host: batch made for another structure");
  cudaStream_t s = (cudaStream_t)stream;
  const int B = bt->n_traj;
  const size_t NS = (size_t)st->n_hier * st->n_state;
  // the stage vectors hold nothing between calls: they stage the host state
  // ([B][n_hier*n_state] complex128 = 16 E bytes <= the 3 E stage elements)
  double2* stage = static_cast<double2*>(bt->acc);
  HOST_CUDA(cudaMemcpyAsync(stage, phi_host, NS * B * 16, cudaMemcpyHostToDevice, s));
  const size_t E = NS * B;
  if (bt->precision == HOPS_PREC_C64)
    k_state_in<float2><<<grid_of(E), 256, 0, s>>>(stage, (float2*)bt->phi, nullptr, B, NS);
  else
    k_state_in<double2><<<grid_of(E), 256, 0, s>>>(stage, (double2*)bt->phi,
                                                   (float2*)bt->phi_lo, B, NS);
  HOST_CUDA(cudaGetLastError());
  const size_t zb = (size_t)B * st->n_mode * 16;
  if (zb) {
    if (zmem_host) HOST_CUDA(cudaMemcpyAsync(bt->zmem, zmem_host, zb, cudaMemcpyHostToDevice, s));
    else HOST_CUDA(cudaMemsetAsync(bt->zmem, 0, zb, s));
  }
  int rc = hops_batch_reset(st, bt, stream);
  if (rc) return rc;
  HOST_CUDA(cudaStreamSynchronize(s));   // the caller may reuse its host buffers on return
  return HOPS_OK;
}

extern "C" int hops_batch_set_noise_host(hops_batch* bt, const float* noise1_host, int32_t n_t1,
                                         const float* noise2_host, int32_t n_t2, void* stream) {
  if (!bt || n_t1 < 0 || n_t2 < 0 || (noise1_host && n_t1 == 0) || (noise2_host && n_t2 == 0))
    return fail(HOPS_EINVAL, "hops_batch_set_noise_host: bad arguments");
  OwnedBatch* ob = reinterpret_cast<OwnedBatch*>(bt);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t rows = (size_t)bt->n_traj * ob->n_lop;
  const size_t b1 = noise1_host ? rows * n_t1 * 8 : 0, b2 = noise2_host ? rows * n_t2 * 8 : 0;
  const size_t b1a = (b1 + 255) & ~(size_t)255;
  if (b1a + b2 > ob->noise_bytes) {
    HOST_CUDA(cudaStreamSynchronize(s));   // the old noise may still be in use
    HOST_CUDA(cudaFree(ob->noise));
    ob->noise = nullptr;
    ob->noise_bytes = 0;
    HOST_CUDA(cudaMalloc(&ob->noise, b1a + b2));
    ob->noise_bytes = b1a + b2;
  }
  unsigned char* p = static_cast<unsigned char*>(ob->noise);
  if (b1) HOST_CUDA(cudaMemcpyAsync(p, noise1_host, b1, cudaMemcpyHostToDevice, s));
  if (b2) HOST_CUDA(cudaMemcpyAsync(p + b1a, noise2_host, b2, cudaMemcpyHostToDevice, s));
  bt->noise1 = b1 ? reinterpret_cast<const float*>(p) : nullptr;
  bt->n_t1 = b1 ? n_t1 : 0;
  bt->noise2 = b2 ? reinterpret_cast<const float*>(p + b1a) : nullptr;
  bt->n_t2 = b2 ? n_t2 : 0;
  HOST_CUDA(cudaStreamSynchronize(s));
  return HOPS_OK;
}

extern "C" int hops_batch_propagate_host(const hops_structure* st, hops_batch* bt, int32_t it0,
                                         int32_t di, int32_t n_steps, double tau_over_hbar,
                                         double* psi_out_host, int32_t* status_host,
                                         void* stream) {
  if (!st || !bt) return fail(HOPS_EINVAL, "hops_batch_propagate_host: null argument");
  int rc = hops_check_propagate_args(st, bt, it0, di, n_steps);
  if (rc) return rc;
  OwnedBatch* ob = reinterpret_cast<OwnedBatch*>(bt);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t need = psi_out_host ? (size_t)n_steps * bt->n_traj * st->n_state : 0;
  if (need > ob->psi_cap) {
    HOST_CUDA(cudaStreamSynchronize(s));
    HOST_CUDA(cudaFree(ob->psi));
    ob->psi = nullptr;
    ob->psi_cap = 0;
    HOST_CUDA(cudaMalloc(&ob->psi, need * 16));
    ob->psi_cap = need;
  }
  rc = hops_rk4_propagate(st, bt, it0, di, n_steps, tau_over_hbar, need ? ob->psi : nullptr,
                          stream);
  if (rc) return rc;
  if (need)
    HOST_CUDA(cudaMemcpyAsync(psi_out_host, ob->psi, need * 16, cudaMemcpyDeviceToHost, s));
  if (status_host)
    HOST_CUDA(cudaMemcpyAsync(status_host, bt->status, (size_t)bt->n_traj * 4,
                              cudaMemcpyDeviceToHost, s));
  HOST_CUDA(cudaStreamSynchronize(s));
  return HOPS_OK;
}

extern "C" int hops_batch_get_state_host(const hops_structure* st, hops_batch* bt,
                                         double* phi_host, double* zmem_host, void* stream) {
  if (!st || !bt) return fail(HOPS_EINVAL, "hops_batch_get_state_host: null argument");
  OwnedBatch* ob = reinterpret_cast<OwnedBatch*>(bt);
  if (ob->n_hier != st->n_hier || ob->n_state != st->n_state)
    return fail(HOPS_EINVAL, "hops_batch_get_state_host: batch made for another structure");
  int rc = hops_batch_settle(st, bt, stream);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int B = bt->n_traj;
  const size_t NS = (size_t)st->n_hier * st->n_state;
  double2* stage = static_cast<double2*>(bt->acc);
  if (phi_host) {
    if (bt->precision == HOPS_PREC_C64)
      k_state_out<float2><<<grid_of(NS * B), 256, 0, s>>>((const float2*)bt->phi, stage, B, NS);
    else
      k_state_out<double2><<<grid_of(NS * B), 256, 0, s>>>((const double2*)bt->phi, stage, B, NS);
    HOST_CUDA(cudaGetLastError());
    HOST_CUDA(cudaMemcpyAsync(phi_host, stage, NS * B * 16, cudaMemcpyDeviceToHost, s));
  }
  if (zmem_host && st->n_mode > 0)
    HOST_CUDA(cudaMemcpyAsync(zmem_host, bt->zmem, (size_t)B * st->n_mode * 16,
                              cudaMemcpyDeviceToHost, s));
  HOST_CUDA(cudaStreamSynchronize(s));
  return HOPS_OK;
}
