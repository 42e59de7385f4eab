// C-ABI implementation of libpfdd_b200.so (declared in include/pfdd_b200.h).
//
// Host side: FP64 set-up of every per-instance constant (what
// FFTW_Slab::setup computes: rotate_stress, frec, stiffness, Bmatrix,
// fft_fftw_slab.cpp:111-119), device buffers, radix plans and twiddle tables,
// and the per-step launch sequence P1 -> P2 -> P3 -> finalize of
// pfdd_kernels.cuh.  Multi-step advances are captured once into a CUDA graph
// per (step count, buffer parity) and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "pfdd_b200.h"
#include "pfdd_kernels.cuh"
#include "pfdd_setup.cuh"

using namespace pfdd;
using namespace pfdd::host;

namespace {

thread_local std::string g_create_error;

// Test hook of the allocation-failure path: PFDD_FAIL_ALLOC_ABOVE=<bytes> in
// the environment makes every device allocation of the library larger than
// that fail as cudaMalloc does when memory runs out (nothing is allocated).
bool alloc_refused(size_t n) {
  const char *e = getenv("PFDD_FAIL_ALLOC_ABOVE");
  return e && *e && n > (size_t)strtoull(e, nullptr, 10);
}

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t alloc(size_t n) {
    if (n && alloc_refused(n)) {
      bytes = 0;
      return cudaErrorMemoryAllocation;
    }
    bytes = n;
    return n ? cudaMalloc(&p, n) : cudaSuccess;
  }
  template <typename T> T *as() const { return reinterpret_cast<T *>(p); }
};

template <typename T> struct Threads;
// plane: whole-plane P1/P3 CTAs; half: each CTA of a split (2-CTA cluster)
// plane; pencil: P2 CTAs.  FP32 defaults were measured on 256x256x128 with
// 12 systems: 256-thread split-plane CTAs at three per SM (80 registers) and
// 256-thread pencil CTAs of at most 107 KB of shared memory at two per SM
// beat 512-thread CTAs at one per SM by 0.3 ms per step.
#ifndef PFDD_HALF_THREADS_F32
#define PFDD_HALF_THREADS_F32 256
#endif
#ifndef PFDD_PENCIL_THREADS_F32
#define PFDD_PENCIL_THREADS_F32 256
#endif
#ifndef PFDD_PENCIL_SMEM_KB
#define PFDD_PENCIL_SMEM_KB 107
#endif
template <> struct Threads<float> {
  static constexpr int plane = 512, half = PFDD_HALF_THREADS_F32, pencil = PFDD_PENCIL_THREADS_F32;
};
template <> struct Threads<double> { static constexpr int plane = 256, half = 256, pencil = 256; };

struct Instance {
  pfdd_instance_desc d;
  int S, F, imag;
  int nx, ny, nz, nzh, nzp, nzs, M;
  int zfused = 1;      // register-resident z passes allowed (PFDD_ZFUSED=0 at creation: off)
  size_t N;
  FftPlan px, py, pz;
  int ccols, fstride, ntiles;
  int sx_n, sy_n;
  bool split = false;  // P1/P3 planes on 2-CTA clusters, half the rows per CTA
  bool merged = false; // in a mixed-size batch: its group runs in the merge class's launches
  size_t smem_plane, smem_update, smem_pencil;
  DevBuf aux;          // Nyquist spectrum of Im xi (IMAG_NYQ)
  DevBuf ppart;        // per-tile partial sums of P2
  Green green;
  Core core;
  StressArgs stress;
  DevBuf xi[2];        // ping-pong real fields [F][N]
  int cur = 0;
  DevBuf spec;         // [F][nx][ny][nzh] complex
  DevBuf partials;     // 2 sums x F * nx planes (x 2 CTAs of a split plane)
  DevBuf stats;        // 2 * cap doubles
  int stats_cap = 0;
  DevBuf small;        // tau[12], sigma[9], dsigma[9], flags[8]
  DevBuf mask, site;
  DevBuf tw_x, tw_y, tw_z, tw_r, tab16;  // twiddles in compute precision, int16 tables
  const int16_t *posM = nullptr, *kx_of = nullptr, *ky_of = nullptr, *kz_of = nullptr, *negy = nullptr,
                *kord = nullptr;
  std::vector<double> hist;  // host copy of the last advance's per-step stats
  int hist_count = 0;
  int group = -1;       // index of the batched group this instance belongs to
  bool advanced = false;  // an advance ran: the device sigma is one increment past its last stress state
  unsigned long long steps_total = 0;  // GL iterations run by advances (checkpoint header)
  // adjoint tape and scratch, kept between calls (checkpoints, segment states,
  // lambda pair, Nyquist carrier of lambda, per-plane gradient sums, their
  // total, final state and carrier); tape_steps > 0 while the tape describes
  // the run that ended at the current state
  DevBuf adj_ck, adj_seg[2], adj_last, adj_lam[2], adj_aux, adj_gpart, adj_acc, adj_fin, adj_finaux;
  DevBuf adj_rspec, adj_raux;   // spectrum and carrier of the segment recomputation
  // strain / stress diagnostics scratch, kept between calls (per-system sums,
  // six strain spectra, six strain fields, FP64 field copies, partial sums)
  DevBuf ss_part, ss_spec6, ss_strain6, ss_e9, ss_s9, ss_fpart;
  int tape_steps = 0, tape_K = 1;
  double *tau() const { return small.as<double>(); }
  double *sigma() const { return small.as<double>() + PFDD_MAXS; }   // sigma[9] then dsigma[9]
  int *flags() const { return reinterpret_cast<int *>(small.as<double>() + PFDD_MAXS + 18); }
  // flags: [0] stop, [1] bad, [2] steps_done, [3] a bounded wait ran out, [4] current xi buffer
  double *an() const { return small.as<double>() + PFDD_MAXS + 22; }  // core model 6 amplitude [4]
  // conductivity sub-problem (pfdd_gpu_cond_*): condxi [2][N], its spectrum
  // [2 fields], the four output spectra, their real fields [4][N], the
  // per-y tables [2][ny] and per-iteration partial sums
  // asynchronous state snapshot (pfdd_gpu_snapshot_begin / _wait): FP64
  // planes on the device, copied to the host on the handle's copy stream
  DevBuf snap;
  cudaEvent_t snap_ready = nullptr, snap_done = nullptr;
  bool snap_pending = false;
  bool cond_on = false;
  DevBuf cond_xi, cond_in, cond_out, cond_real, cond_tab, cond_part;
  double cond_El = 0.0, cond_eps0 = 0.0, cond_dt = 0.0;
  const void *site_arg = nullptr;  // `site` argument of the update kernels
};

}  // namespace

// Instances whose grid, slip systems, material, core model and carrier mode
// agree run as one group: one launch per kernel per step for all of them.
struct Group {
  std::vector<int> members;
  DevBuf table;   // InstPtrs[members.size()]
};

// Groups of one merge class (everything equal but the grid size) that run
// in one launch per pass (k_*_multi); the device tables hold each group's
// arguments, MultiLaunch the CTA prefix of each group.
struct MergeClass {
  std::vector<int> groups;
  DevBuf ptab, pentab, ftab;   // MultiPlaneGroup[], MultiPencilGroup[], MultiFinalGroup[]
  MultiLaunch mp{}, mpe{}, mf{};
  unsigned plane_ctas = 0, pencil_ctas = 0, insts = 0;
  size_t smem_plane = 0, smem_pencil = 0;
  int S = 0;
};

struct GraphKey {
  int steps;
  int states;   // 0: steps of the current stress state; k > 0: k whole stress states of `steps` steps
  double tol;
  bool operator<(const GraphKey &o) const {
    if (steps != o.steps) return steps < o.steps;
    if (states != o.states) return states < o.states;
    return tol < o.tol;
  }
};

struct pfdd_gpu {
  int precision = PFDD_FP64;
  int device = 0;
  pfdd_options opt{};
  std::vector<std::unique_ptr<Instance>> inst;
  std::vector<Group> groups;
  std::vector<MergeClass> merges;  // mixed-size batches
  std::vector<int> group_merge;    // per group: its merge class, or -1 (own launches)
  std::map<GraphKey, cudaGraphExec_t> graphs;   // K-step launch sequences, replayed by advance
  cudaStream_t stream = nullptr;      // stream in use
  cudaStream_t own_stream = nullptr;  // stream created by the handle
  DevBuf staging;                     // FP64 host<->device staging, kept across calls
  cudaStream_t copy_stream = nullptr; // device-to-host snapshots, beside the stepping stream
  cudaStream_t side_stream = nullptr; // the adjoint's segment recomputation, beside its backward steps
  std::string err;
  size_t device_bytes = 0;
  int nsm = 148;                      // SMs of the device (grid sizing)
  // a create that fails part-way still releases its stream (device buffers
  // free themselves)
  ~pfdd_gpu() {
    if (own_stream) cudaStreamDestroy(own_stream);
  }
};

namespace {

pfdd_status fail(pfdd_gpu *h, pfdd_status code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  else g_create_error = buf;
  return code;
}

#define CUDA_TRY(h, call)                                                                   \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(h, e_ == cudaErrorMemoryAllocation ? PFDD_ENOMEM : PFDD_ECUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                       \
  } while (0)

// Error words of an instance, cleared where a call that steps or transforms
// starts (a reported divergence or timeout does not stick to the handle), and
// the stall test switch of the bounded-wait path (flags[5]): with
// PFDD_STALL_BULK_WAITS=1 in the environment, every plane-pass CTA's copy
// barrier withholds one arrival, so its first wait runs out after
// kStallWaitNs, the CTA waits for its copies to land, sets the timeout word
// and abandons the plane; the call returns PFDD_ETIMEOUT and the state is
// undefined until the next set_state.  Read at each such call.
int stall_requested() {
  const char *e = getenv("PFDD_STALL_BULK_WAITS");
  return (e && atoi(e) != 0) ? 1 : 0;
}
#define ARM_FLAGS(h, I)                                                                      \
  do {                                                                                       \
    CUDA_TRY(h, cudaMemsetAsync((I).flags() + 1, 0, sizeof(int), (h)->stream));             \
    CUDA_TRY(h, cudaMemsetAsync((I).flags() + 3, 0, sizeof(int), (h)->stream));             \
    CUDA_TRY(h, cudaMemsetAsync((I).flags() + 5, stall_requested(), sizeof(int), (h)->stream)); \
  } while (0)

template <typename T> size_t csize() { return sizeof(cx<T>); }

// Grow a kept scratch buffer to `bytes` (after the stream's earlier work).
cudaError_t grow(cudaStream_t st, DevBuf &b, size_t bytes) {
  if (b.p && b.bytes >= bytes) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  b.release();
  return b.alloc(bytes);
}

template <typename T>
pfdd_status upload_table(pfdd_gpu *h, DevBuf &dst, const std::vector<double> &tw) {
  std::vector<T> t(tw.size());
  for (size_t i = 0; i < tw.size(); ++i) t[i] = (T)tw[i];
  CUDA_TRY(h, dst.alloc(t.size() * sizeof(T)));
  CUDA_TRY(h, cudaMemcpy(dst.p, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice));
  h->device_bytes += dst.bytes;
  return PFDD_OK;
}

template <typename T>
pfdd_status upload_twiddles(pfdd_gpu *h, DevBuf &dst, int n, int count) {
  std::vector<double> tw;
  twiddles(n, count, tw);
  return upload_table<T>(h, dst, tw);
}

// x-pencil tile of cc (ky, kz) columns: narrowest width is one 16-byte row
// chunk; the field stride is padded so consecutive fields start cc columns
// apart in the 32 shared-memory banks (the x FFT walks columns, then fields,
// across a warp); the tile's shared memory holds the fields, the x twiddles,
// reduction scratch, wave-vector parts (x slots and the tile's columns), the
// columns' slots and the Nyquist snapshot.
template <typename T> int pencil_cmin() { return (int)(16 / sizeof(cx<T>)) > 1 ? (int)(16 / sizeof(cx<T>)) : 1; }

template <typename T> int pencil_fstride(const Instance &I, int cc) {
  using C = cx<T>;
  const int wpc = (int)(sizeof(C) / 4);
  const int target = (cc * wpc) % 32;
  for (int pad = 0; pad < 64; ++pad)
    if ((pad * sizeof(C)) % 16 == 0 && (((size_t)I.nx * cc + pad) * wpc) % 32 == (size_t)target)
      return I.nx * cc + pad;
  return I.nx * cc;
}

template <typename T> size_t pencil_smem(const Instance &I, int cc) {
  using C = cx<T>;
  return ((size_t)I.F * pencil_fstride<T>(I, cc) + (size_t)I.nx) * sizeof(C) + 64 * sizeof(double) +
         ((size_t)I.nx + 2 * (size_t)cc) * sizeof(V4<T>) + 2 * (size_t)((cc + 3) & ~3) * sizeof(int) +
         (size_t)cc * I.S * sizeof(C);
}

template <typename T>
pfdd_status setup_instance(pfdd_gpu *h, Instance &I) {
  const pfdd_instance_desc &d = I.d;
  using C = cx<T>;
  pfdd_status st;
  if ((st = upload_twiddles<T>(h, I.tw_x, I.nx, I.nx))) return st;
  if (I.split) {
    // W_ny^m (m < ny/2) of the cross-CTA stage, then W_{ny/2}^m of the local stages
    std::vector<double> tw, twh;
    twiddles(I.ny, I.ny / 2, tw);
    twiddles(I.ny / 2, I.ny / 2, twh);
    tw.insert(tw.end(), twh.begin(), twh.end());
    if ((st = upload_table<T>(h, I.tw_y, tw))) return st;
  } else if ((st = upload_twiddles<T>(h, I.tw_y, I.ny, I.ny))) {
    return st;
  }
  if ((st = upload_twiddles<T>(h, I.tw_z, I.M, I.M))) return st;
  if ((st = upload_twiddles<T>(h, I.tw_r, I.nz, I.M))) return st;

  // int16 tables: posM[M], kx_of[nx], ky_of[ny], kz_of[nzp], negy[ny], kord[M/2]
  std::vector<int> pz = positions(I.pz), px = positions(I.px), py = positions(I.py);
  std::vector<int16_t> tab(I.M + I.nx + I.ny + I.nzp + I.ny + I.M / 2, 0);
  int16_t *t_posM = tab.data(), *t_kx = t_posM + I.M, *t_ky = t_kx + I.nx, *t_kz = t_ky + I.ny;
  neg_slots(I.ny, I.split, py.data(), t_kz + I.nzp);
  unpack_order(pz.data(), I.M, t_kz + I.nzp + I.ny);
  for (int k = 0; k < I.M; ++k) t_posM[k] = (int16_t)pz[k];
  for (int k = 0; k < I.nx; ++k) t_kx[px[k]] = (int16_t)k;
  if (I.split) {
    // rank r of a split plane holds ky = r + 2 k at the slots of the ny/2 plan
    const int nyh = I.ny / 2;
    for (int r = 0; r < 2; ++r)
      for (int k = 0; k < nyh; ++k) t_ky[r * nyh + py[k]] = (int16_t)(r + 2 * k);
  } else {
    for (int k = 0; k < I.ny; ++k) t_ky[py[k]] = (int16_t)k;
  }
  for (int k = 0; k < I.M; ++k) t_kz[pz[k]] = (int16_t)k;
  t_kz[I.M] = (int16_t)I.M;
  I.sx_n = px[I.nx / 2];
  if (I.split) {
    const int r = (I.ny / 2) % 2;
    I.sy_n = r * (I.ny / 2) + py[(I.ny / 2 - r) / 2];
  } else {
    I.sy_n = py[I.ny / 2];
  }
  CUDA_TRY(h, I.tab16.alloc(tab.size() * sizeof(int16_t)));
  CUDA_TRY(h, cudaMemcpy(I.tab16.p, tab.data(), tab.size() * sizeof(int16_t), cudaMemcpyHostToDevice));
  h->device_bytes += I.tab16.bytes;
  const int16_t *base = I.tab16.as<int16_t>();
  I.posM = base;
  I.kx_of = base + I.M;
  I.ky_of = I.kx_of + I.nx;
  I.kz_of = I.ky_of + I.ny;
  I.negy = I.kz_of + I.nzp;
  I.kord = I.negy + I.ny;

  const size_t fieldN = (size_t)I.F * I.N;
  for (int b = 0; b < 2; ++b) {
    CUDA_TRY(h, I.xi[b].alloc(fieldN * sizeof(T)));
    CUDA_TRY(h, cudaMemset(I.xi[b].p, 0, fieldN * sizeof(T)));
    h->device_bytes += I.xi[b].bytes;
  }
  CUDA_TRY(h, I.spec.alloc((size_t)I.F * I.nx * I.ny * I.nzp * sizeof(C)));
  h->device_bytes += I.spec.bytes;
  CUDA_TRY(h, I.partials.alloc(4 * (size_t)I.F * I.nx * sizeof(double)));   // 2 sums x 2 CTAs of a split plane
  h->device_bytes += I.partials.bytes;
  CUDA_TRY(h, I.small.alloc((PFDD_MAXS + 26) * sizeof(double)));
  CUDA_TRY(h, cudaMemset(I.small.p, 0, (PFDD_MAXS + 26) * sizeof(double)));
  double sig18[18];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      sig18[3 * i + j] = d.sigma[i][j];
      sig18[9 + 3 * i + j] = d.dsigma[i][j];
    }
  CUDA_TRY(h, cudaMemcpy(I.sigma(), sig18, sizeof sig18, cudaMemcpyHostToDevice));

  if (d.xo) {
    std::vector<uint8_t> m((size_t)I.S * I.N);
    for (size_t i = 0; i < m.size(); ++i) m[i] = d.xo[i] != 0.0;
    CUDA_TRY(h, I.mask.alloc(m.size()));
    CUDA_TRY(h, cudaMemcpy(I.mask.p, m.data(), m.size(), cudaMemcpyHostToDevice));
    h->device_bytes += I.mask.bytes;
  }
  if (d.core_flag == PFDD_CORE_MPEA || d.core_flag == PFDD_CORE_SINE_FIELD) {
    if (!d.site_gsfe) return fail(h, PFDD_EINVAL, "core model %d needs site_gsfe", d.core_flag);
    std::vector<T> sv((size_t)I.S * I.N);
    for (size_t i = 0; i < sv.size(); ++i) sv[i] = (T)d.site_gsfe[i];
    CUDA_TRY(h, I.site.alloc(sv.size() * sizeof(T)));
    CUDA_TRY(h, cudaMemcpy(I.site.p, sv.data(), sv.size() * sizeof(T), cudaMemcpyHostToDevice));
    h->device_bytes += I.site.bytes;
  }
  // core model 6 reads its per-state amplitude (An' pi, An') where the
  // per-site models read their field: FP64 at an(), FP32 after them
  I.site_arg = I.site.p;
  if (d.core_flag == PFDD_CORE_USFE_ANGLE)
    I.site_arg = sizeof(T) == 8 ? (const void *)I.an() : (const void *)(I.an() + 2);
  if (d.non_schmid && I.S > 3)
    return fail(h, PFDD_EINVAL, "non-Schmid stress needs n_slip <= 3 (resolSS_non_Schmid tables)");

  // shared-memory budgets
  I.smem_plane = PlaneSmem<C>::bytes(I.split ? I.ny / 2 : I.ny, I.ny, I.nzs, I.M);
  I.smem_update = I.smem_plane;
  const size_t limit = 227 * 1024;
  if (I.smem_update > limit)
    return fail(h, PFDD_EUNSUPPORTED, "x-plane of %dx%d does not fit shared memory in this precision", I.ny, I.nz);
  const size_t ncols = (size_t)I.ny * I.nzp;
  const int cmin = pencil_cmin<T>();
  auto fstride_for = [&](int cc) { return pencil_fstride<T>(I, cc); };
  auto pencil_bytes = [&](int cc) { return pencil_smem<T>(I, cc); };
  int cc = 32;
  // widest tile that fits the budget and still gives every SM two tiles
  while (cc > cmin && (ncols % cc || pencil_bytes(cc) > PFDD_PENCIL_SMEM_KB * 1024 ||
                       ncols / cc < 2 * (size_t)h->nsm))
    cc >>= 1;
  if (ncols % cc || pencil_bytes(cc) > limit)
    return fail(h, PFDD_EUNSUPPORTED, "x-pencil of %d x %d fields does not fit shared memory", I.nx, I.F);
  I.ccols = cc;
  I.fstride = fstride_for(cc);
  I.ntiles = (int)(ncols / cc);
  I.smem_pencil = pencil_bytes(cc);
  if (I.imag == IMAG_NYQ) {
    const size_t na = (size_t)I.S * ((size_t)I.nx * I.ny + (size_t)I.nx * I.M + (size_t)I.ny * I.M);
    CUDA_TRY(h, I.aux.alloc(na * sizeof(C)));
    CUDA_TRY(h, cudaMemset(I.aux.p, 0, na * sizeof(C)));
    h->device_bytes += I.aux.bytes;
    CUDA_TRY(h, I.ppart.alloc(2 * (size_t)I.ntiles * sizeof(double)));
    h->device_bytes += I.ppart.bytes;
  }

  build_green(d, I.green);
  if (!build_core(d, I.core)) return fail(h, PFDD_EUNSUPPORTED, "core model %d not supported", d.core_flag);
  build_stress(d, I.stress);
  return PFDD_OK;
}

template <typename T>
void fill_plane_args(const Instance &I, PlaneArgs &pa) {
  pa.py = I.py; pa.pz = I.pz;
  pa.nx = I.nx; pa.ny = I.ny; pa.nz = I.nz; pa.nzh = I.nzh; pa.nzp = I.nzp; pa.nzs = I.nzs; pa.M = I.M;
  pa.S = I.S; pa.F = I.F;
  pa.tw_y = I.tw_y.p; pa.tw_z = I.tw_z.p; pa.tw_r = I.tw_r.p;
  pa.posM = I.posM;
  pa.negy = I.negy;
  pa.kord = I.kord;
  set_plane_divisors<T>(pa, I.split ? I.ny / 2 : I.ny);
  pa.zfused = I.zfused;
}

template <typename T>
pfdd_status set_smem_attrs(pfdd_gpu *h, size_t plane, size_t upd, size_t pencil) {
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half, NC = Threads<T>::pencil;
  CUDA_TRY(h, raise_smem_limit(k_fwd_planes<T, NP, false>, plane));
  CUDA_TRY(h, raise_smem_limit(k_fwd_planes<T, NH, true>, plane));
  CUDA_TRY(h, raise_smem_limit(k_inv_update<T, NP, false>, upd));
  CUDA_TRY(h, raise_smem_limit(k_inv_update<T, NH, true>, upd));
  cudaError_t pe_err = cudaSuccess;
  for (int sc : {0, 2, 3, 12})
    with_pencil_sc(sc, [&](auto SCc) {
      constexpr int SC = decltype(SCc)::value;
      if (pe_err == cudaSuccess) pe_err = raise_smem_limit(k_xpencil<T, NC, SC>, pencil);
      if (pe_err == cudaSuccess) pe_err = raise_smem_limit(k_xpencil_tab<T, NC, SC>, pencil);
    });
  CUDA_TRY(h, pe_err);
  CUDA_TRY(h, raise_smem_limit(k_fwd_planes_tab<T, NP, false>, plane));
  CUDA_TRY(h, raise_smem_limit(k_fwd_planes_tab<T, NH, true>, plane));
  CUDA_TRY(h, raise_smem_limit(k_inv_update_tab<T, NP, false>, upd));
  CUDA_TRY(h, raise_smem_limit(k_inv_update_tab<T, NH, true>, upd));
  CUDA_TRY(h, raise_smem_limit(k_step_planes<T, NP, false>, upd));
  CUDA_TRY(h, raise_smem_limit(k_step_planes<T, NH, true>, upd));
  CUDA_TRY(h, raise_smem_limit(k_step_planes_tab<T, NP, false>, upd));
  CUDA_TRY(h, raise_smem_limit(k_adj_planes<T, NP, false>, upd));
  CUDA_TRY(h, raise_smem_limit(k_adj_planes<T, NH, true>, upd));
  CUDA_TRY(h, raise_smem_limit(k_step_planes_tab<T, NH, true>, upd));
  return PFDD_OK;
}

// P2 of one instance, with the contraction unrolled for its slip-system count
template <typename T>
void launch_pencil(const Instance &I, cudaStream_t st, cx<T> *spec, const PencilArgs &pe, const int *stop) {
  constexpr int NC = Threads<T>::pencil;
  with_pencil_sc(I.S, [&](auto SCc) {
    k_xpencil<T, NC, decltype(SCc)::value><<<I.ntiles, NC, I.smem_pencil, st>>>(spec, pe, stop);
  });
}

// Launch with an optional 2-CTA cluster (split planes).
template <typename K, typename... Args>
void launch_pair(K kernel, dim3 grid, int nt, size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(nt, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

// P1 of one instance (grid.x = planes) or of a group (grid.y = instances)
template <typename T>
void launch_fwd(const Instance &I, cudaStream_t st, const T *xin, cx<T> *spec, const PlaneArgs &pa,
                const int *stop, int *err) {
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half;
  const unsigned planes = (unsigned)(I.F * I.nx);
  if (I.split) launch_pair(k_fwd_planes<T, NH, true>, dim3(2 * planes), NH, I.smem_plane, st, xin, spec, pa, stop, err);
  else k_fwd_planes<T, NP, false><<<planes, NP, I.smem_plane, st>>>(xin, spec, pa, stop, err);
}

template <typename T>
void launch_fwd_tab(const Instance &L, unsigned B, cudaStream_t st, const InstPtrs *tab, const PlaneArgs &pa) {
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half;
  const unsigned planes = (unsigned)(L.F * L.nx);
  if (L.split) launch_pair(k_fwd_planes_tab<T, NH, true>, dim3(2 * planes, B), NH, L.smem_plane, st, tab, pa);
  else k_fwd_planes_tab<T, NP, false><<<dim3(planes, B), NP, L.smem_plane, st>>>(tab, pa);
}

// P3 of one instance (any pass)
template <typename T>
void launch_inv(const Instance &I, unsigned planes, cudaStream_t st, const cx<T> *spec, const T *xin, T *xout,
                const PlaneArgs &pa, const UpdateArgs &ua, double *partials) {
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half;
  if (I.split)
    launch_pair(k_inv_update<T, NH, true>, dim3(2 * planes), NH, I.smem_update, st, spec, xin, xout, pa, ua, partials);
  else k_inv_update<T, NP, false><<<planes, NP, I.smem_update, st>>>(spec, xin, xout, pa, ua, partials);
}


// Fused plane pass of a group (P3 of this step + P1 of the next when fwd)
template <typename T>
void launch_step_tab(const Instance &L, unsigned B, cudaStream_t st, const InstPtrs *tab, const PlaneArgs &pa,
                     const UpdateArgs &ua, bool fwd) {
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half;
  const unsigned planes = (unsigned)(L.F * L.nx);
  if (L.split)
    launch_pair(k_step_planes_tab<T, NH, true>, dim3(2 * planes, B), NH, L.smem_update, st, tab, pa, ua, (int)fwd);
  else k_step_planes_tab<T, NP, false><<<dim3(planes, B), NP, L.smem_update, st>>>(tab, pa, ua, (int)fwd);
}

// Buffers of one adjoint iteration: lambda in and out, the forward state it
// linearises about, the Nyquist carrier of lambda and the gradient partials
// (P1 and P2 are those of the forward step: the elastic operator is
// self-adjoint).
struct AdjointPass {
  void *lam_in, *lam_out;
  const void *xfwd;
  void *aux;
  double *gpart;
};

// One GL iteration (or, with adj, one adjoint iteration) of instance I whose
// spectrum is current, i.e. opened by launch_fwd or left by the previous fused
// plane pass: P2, the fused plane pass (fwd: also the next iteration's
// spectrum) and, for forward steps, the reduction.
// Forward steps may read and write explicit state buffers (fin/fout, the
// adjoint's tape) and leave out the reduction (stats = false).
// spec_buf / aux_buf: another spectrum and Nyquist carrier than the
// instance's (the adjoint recomputes segments beside its backward steps).
template <typename T>
void enqueue_step_fused(Instance &I, cudaStream_t st, bool fwd, const AdjointPass *adj = nullptr,
                        const void *fin = nullptr, void *fout = nullptr, bool stats = true,
                        void *spec_buf = nullptr, void *aux_buf = nullptr) {
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half;
  PlaneArgs pa;
  fill_plane_args<T>(I, pa);
  int *flags = I.flags();
  const T *xin = adj ? static_cast<const T *>(adj->lam_in)
                     : (fin ? static_cast<const T *>(fin) : I.xi[I.cur].as<T>());
  T *xout = adj ? static_cast<T *>(adj->lam_out) : (fout ? static_cast<T *>(fout) : I.xi[I.cur ^ 1].as<T>());
  cx<T> *spec = spec_buf ? static_cast<cx<T> *>(spec_buf) : I.spec.as<cx<T>>();
  const int planes = I.F * I.nx;
  PencilArgs pe{};
  pe.px = I.px;
  pe.nx = I.nx; pe.ny = I.ny; pe.nz = I.nz; pe.nzh = I.nzh; pe.nzp = I.nzp; pe.M = I.M;
  pe.S = I.S; pe.F = I.F; pe.imag = I.imag;
  pe.ncols = I.ny * I.nzp;
  pe.ccols = I.ccols;
  pe.tw_x = I.tw_x.p;
  pe.kx_of = I.kx_of; pe.ky_of = I.ky_of; pe.kz_of = I.kz_of;
  pe.mode = PASS_STEP;
  pe.fstride = I.fstride;
  pe.aux = adj ? adj->aux : (aux_buf ? aux_buf : I.aux.p);
  pe.sx_n = I.sx_n; pe.sy_n = I.sy_n;
  pe.cd = I.d.cd_dt;
  pe.partials = (I.imag == IMAG_NYQ && !adj && stats) ? I.ppart.as<double>() : nullptr;
  pe.g = I.green;
  set_pencil_divisors<T>(pe);
  launch_pencil<T>(I, st, spec, pe, flags);
  UpdateArgs ua;
  memset(&ua, 0, sizeof ua);
  ua.nx = I.nx; ua.ny = I.ny; ua.nz = I.nz; ua.nzh = I.nzh; ua.nzp = I.nzp; ua.S = I.S; ua.F = I.F;
  ua.cd = I.d.cd_dt;
  ua.invN = 1.0 / (double)I.N;
  ua.core = I.core;
  ua.tau = I.tau();
  ua.mask = I.mask.as<uint8_t>();
  ua.site = I.site_arg;
  ua.stop = flags;
  ua.err = flags + 3;
  ua.mode = adj ? PASS_ADJOINT : PASS_STEP;
  ua.xfwd = adj ? adj->xfwd : nullptr;
  ua.gpart = adj ? adj->gpart : nullptr;
  double *partials = I.partials.as<double>();
  if (adj) {
    if (I.split)
      launch_pair(k_adj_planes<T, NH, true>, dim3(2 * planes), NH, I.smem_update, st, spec, xin, xout, pa, ua,
                  partials, (int)fwd);
    else k_adj_planes<T, NP, false><<<planes, NP, I.smem_update, st>>>(spec, xin, xout, pa, ua, partials, (int)fwd);
    return;
  }
  if (I.split)
    launch_pair(k_step_planes<T, NH, true>, dim3(2 * planes), NH, I.smem_update, st, spec, xin, xout, pa, ua,
                partials, (int)fwd);
  else k_step_planes<T, NP, false><<<planes, NP, I.smem_update, st>>>(spec, xin, xout, pa, ua, partials, (int)fwd);
  if (!stats) return;
  const bool nyq = I.imag == IMAG_NYQ;
  // a split plane's CTAs write a partial each (plane_sum_slots)
  k_finalize<<<1, 1024, 0, st>>>(partials, I.split ? 2 * planes : planes, I.stats.as<double>(), 0, 0.0, flags,
                                 flags + 1, flags + 2, nyq ? I.ppart.as<double>() : nullptr, nyq ? I.ntiles : 0,
                                 1.0 / (double)I.N);
}

// ------------------------------------------------------------ batched groups
bool same_group(const Instance &a, const Instance &b) {
  const pfdd_instance_desc &x = a.d, &y = b.d;
  if (a.nx != b.nx || a.ny != b.ny || a.nz != b.nz || a.S != b.S || a.F != b.F || a.imag != b.imag) return false;
  if (x.core_flag != y.core_flag || x.C44 != y.C44 || x.C12 != y.C12 || x.C11 != y.C11 || x.dslip != y.dslip ||
      x.b != y.b || x.cd_dt != y.cd_dt || x.isf != y.isf || x.usf != y.usf || x.An != y.An)
    return false;
  if (memcmp(x.four, y.four, sizeof x.four) || memcmp(x.prim, y.prim, sizeof x.prim) ||
      memcmp(x.xn, y.xn, sizeof(double) * 3 * a.S) || memcmp(x.xb, y.xb, sizeof(double) * 3 * a.S) ||
      memcmp(x.c, y.c, sizeof x.c) || memcmp(x.aa, y.aa, sizeof x.aa) || memcmp(x.bb, y.bb, sizeof x.bb))
    return false;
  // one StressArgs serves the whole group
  if ((x.non_schmid != 0) != (y.non_schmid != 0) || x.angle_to_110 != y.angle_to_110 || x.w1 != y.w1 ||
      x.w2 != y.w2 || x.w3 != y.w3 || memcmp(x.usfe_fit, y.usfe_fit, sizeof x.usfe_fit))
    return false;
  if ((a.mask.p == nullptr) != (b.mask.p == nullptr) || (a.site.p == nullptr) != (b.site.p == nullptr)) return false;
  return true;
}

// Instances that differ in nothing but the grid size (slip systems, carrier,
// material, core model, stress projections, mask and GSFE-field presence):
// their groups can share the mixed-size launches.
bool same_class(const Instance &a, const Instance &b) {
  if (a.S != b.S || a.F != b.F || a.imag != b.imag || a.split || b.split) return false;
  const pfdd_instance_desc &x = a.d, &y = b.d;
  if (x.core_flag != y.core_flag || x.C44 != y.C44 || x.C12 != y.C12 || x.C11 != y.C11 || x.dslip != y.dslip ||
      x.b != y.b || x.cd_dt != y.cd_dt || x.isf != y.isf || x.usf != y.usf || x.An != y.An)
    return false;
  if (memcmp(x.four, y.four, sizeof x.four) || memcmp(x.prim, y.prim, sizeof x.prim) ||
      memcmp(x.xn, y.xn, sizeof(double) * 3 * a.S) || memcmp(x.xb, y.xb, sizeof(double) * 3 * a.S) ||
      memcmp(x.c, y.c, sizeof x.c) || memcmp(x.aa, y.aa, sizeof x.aa) || memcmp(x.bb, y.bb, sizeof x.bb))
    return false;
  if ((x.non_schmid != 0) != (y.non_schmid != 0) || x.angle_to_110 != y.angle_to_110 || x.w1 != y.w1 ||
      x.w2 != y.w2 || x.w3 != y.w3 || memcmp(x.usfe_fit, y.usfe_fit, sizeof x.usfe_fit))
    return false;
  return (a.mask.p == nullptr) == (b.mask.p == nullptr) && (a.site.p == nullptr) == (b.site.p == nullptr);
}

template <typename T> const GreenT<T> &green_host(const Green &g);
template <> const GreenT<double> &green_host<double>(const Green &g) { return g.d; }
template <> const GreenT<float> &green_host<float>(const Green &g) { return g.f; }

// x-pencil arguments of instance L's group (the tile width is the group's)
template <typename T>
void group_pencil_args(const Instance &L, PencilArgs &pe) {
  pe = PencilArgs{};
  pe.px = L.px;
  pe.nx = L.nx; pe.ny = L.ny; pe.nz = L.nz; pe.nzh = L.nzh; pe.nzp = L.nzp; pe.M = L.M;
  pe.S = L.S; pe.F = L.F; pe.imag = L.imag;
  pe.ncols = L.ny * L.nzp;
  pe.ccols = L.ccols;
  pe.tw_x = L.tw_x.p;
  pe.kx_of = L.kx_of; pe.ky_of = L.ky_of; pe.kz_of = L.kz_of;
  pe.mode = PASS_STEP;
  pe.fstride = L.fstride;
  pe.sx_n = L.sx_n; pe.sy_n = L.sy_n;
  pe.cd = L.d.cd_dt;
  pe.g = L.green;
  set_pencil_divisors<T>(pe);
}

// update arguments of instance L's group stepping (per-instance pointers come
// from the group table)
void group_update_args(const Instance &L, UpdateArgs &ua) {
  memset(&ua, 0, sizeof ua);
  ua.nx = L.nx; ua.ny = L.ny; ua.nz = L.nz; ua.nzh = L.nzh; ua.nzp = L.nzp; ua.S = L.S; ua.F = L.F;
  ua.cd = L.d.cd_dt;
  ua.invN = 1.0 / (double)L.N;
  ua.core = L.core;
  ua.mode = PASS_STEP;
}

template <typename T>
pfdd_status build_merges_t(pfdd_gpu *h) {
  constexpr int NC = Threads<T>::pencil;
  h->merges.clear();
  h->group_merge.assign(h->groups.size(), -1);
  std::vector<std::vector<int>> cls;
  for (size_t gi = 0; gi < h->groups.size(); ++gi) {
    const Instance &L = *h->inst[h->groups[gi].members[0]];
    if (!L.merged || L.split) continue;
    int c = -1;
    for (size_t k = 0; k < cls.size() && c < 0; ++k)
      if ((int)cls[k].size() < kMaxMerged && same_class(*h->inst[h->groups[cls[k][0]].members[0]], L)) c = (int)k;
    if (c < 0) {
      cls.emplace_back();
      c = (int)cls.size() - 1;
    }
    cls[c].push_back((int)gi);
  }
  for (auto &gl : cls) {
    if (gl.size() < 2) continue;
    h->merges.emplace_back();
    MergeClass &mc = h->merges.back();
    mc.groups = gl;
    const int n = (int)gl.size();
    std::vector<MultiPlaneGroup> pg(n);
    std::vector<MultiPencilGroup> peg(n);
    std::vector<MultiFinalGroup> fg(n);
    mc.mp.ngroups = mc.mpe.ngroups = mc.mf.ngroups = n;
    unsigned pc = 0, pec = 0, ic = 0;
    for (int k = 0; k < n; ++k) {
      const Group &G = h->groups[gl[k]];
      const Instance &L = *h->inst[G.members[0]];
      const unsigned B = (unsigned)G.members.size();
      fill_plane_args<T>(L, pg[k].a);
      group_update_args(L, pg[k].u);
      pg[k].tab = static_cast<const InstPtrs *>(G.table.p);
      pg[k].per_member = L.F * L.nx;
      group_pencil_args<T>(L, peg[k].a);
      peg[k].tab = pg[k].tab;
      peg[k].per_member = L.ntiles;
      fg[k].tab = pg[k].tab;
      fg[k].nparts = L.F * L.nx;
      fg[k].nparts2 = L.imag == IMAG_NYQ ? L.ntiles : 0;
      fg[k].scale2 = 1.0 / (double)L.N;
      mc.mp.starts[k] = (int)pc;
      mc.mpe.starts[k] = (int)pec;
      mc.mf.starts[k] = (int)ic;
      pc += B * (unsigned)pg[k].per_member;
      pec += B * (unsigned)L.ntiles;
      ic += B;
      mc.smem_plane = std::max(mc.smem_plane, L.smem_update);
      mc.smem_pencil = std::max(mc.smem_pencil, L.smem_pencil);
      mc.S = L.S;
    }
    mc.mp.starts[n] = (int)pc;
    mc.mpe.starts[n] = (int)pec;
    mc.mf.starts[n] = (int)ic;
    mc.plane_ctas = pc;
    mc.pencil_ctas = pec;
    mc.insts = ic;
    CUDA_TRY(h, mc.ptab.alloc(n * sizeof(MultiPlaneGroup)));
    CUDA_TRY(h, cudaMemcpy(mc.ptab.p, pg.data(), n * sizeof(MultiPlaneGroup), cudaMemcpyHostToDevice));
    CUDA_TRY(h, mc.pentab.alloc(n * sizeof(MultiPencilGroup)));
    CUDA_TRY(h, cudaMemcpy(mc.pentab.p, peg.data(), n * sizeof(MultiPencilGroup), cudaMemcpyHostToDevice));
    CUDA_TRY(h, mc.ftab.alloc(n * sizeof(MultiFinalGroup)));
    CUDA_TRY(h, cudaMemcpy(mc.ftab.p, fg.data(), n * sizeof(MultiFinalGroup), cudaMemcpyHostToDevice));
    CUDA_TRY(h, raise_smem_limit(k_step_planes_multi<T, 256>, mc.smem_plane));
    CUDA_TRY(h, raise_smem_limit(k_fwd_planes_multi<T, 256>, mc.smem_plane));
    cudaError_t e = cudaSuccess;
    with_pencil_sc(mc.S, [&](auto SCc) {
      constexpr int SC = decltype(SCc)::value;
      e = raise_smem_limit(k_xpencil_multi<T, NC, SC>, mc.smem_pencil);
    });
    CUDA_TRY(h, e);
    for (int g : gl) h->group_merge[g] = (int)h->merges.size() - 1;
  }
  return PFDD_OK;
}

pfdd_status build_merges(pfdd_gpu *h) {
  return h->precision == PFDD_FP64 ? build_merges_t<double>(h) : build_merges_t<float>(h);
}

// Write every group's InstPtrs table (after any per-instance buffer changes).
pfdd_status refresh_tables(pfdd_gpu *h) {
  for (auto &G : h->groups) {
    std::vector<InstPtrs> t(G.members.size());
    for (size_t k = 0; k < G.members.size(); ++k) {
      Instance &I = *h->inst[G.members[k]];
      InstPtrs &p = t[k];
      p.xi[0] = I.xi[0].p;
      p.xi[1] = I.xi[1].p;
      p.spec = I.spec.p;
      p.aux = I.aux.p;
      p.ppart = I.imag == IMAG_NYQ ? I.ppart.as<double>() : nullptr;
      p.partials = I.partials.as<double>();
      p.tau = I.tau();
      p.sigma = I.sigma();
      p.flags = I.flags();
      p.stats = I.stats.as<double>();
      p.stats_cap = I.stats_cap;
      p.mask = I.mask.as<uint8_t>();
      p.site = I.site_arg;
      p.an = I.an();
    }
    if (!G.table.p) CUDA_TRY(h, G.table.alloc(t.size() * sizeof(InstPtrs)));
    CUDA_TRY(h, cudaMemcpy(G.table.p, t.data(), t.size() * sizeof(InstPtrs), cudaMemcpyHostToDevice));
  }
  // the mixed-size launches read tile widths and buffer sizes from their tables
  return build_merges(h);
}

void build_groups(pfdd_gpu *h) {
  h->groups.clear();
  for (size_t i = 0; i < h->inst.size(); ++i) {
    Instance &I = *h->inst[i];
    int g = -1;
    for (size_t k = 0; k < h->groups.size() && g < 0; ++k)
      if (same_group(*h->inst[h->groups[k].members[0]], I)) g = (int)k;
    if (g < 0) {
      h->groups.emplace_back();
      g = (int)h->groups.size() - 1;
    }
    h->groups[g].members.push_back((int)i);
    I.group = g;
  }
}

// The forward pass (P1) that opens a run of steps of group G: every later
// step's spectrum comes from the previous step's fused plane pass.
template <typename T>
void enqueue_group_open(Instance &L, const Group &G, cudaStream_t st) {
  PlaneArgs pa;
  fill_plane_args<T>(L, pa);
  launch_fwd_tab<T>(L, (unsigned)G.members.size(), st, static_cast<const InstPtrs *>(G.table.p), pa);
}

// One GL iteration of every instance of group G whose spectrum is current
// (3 launches: P2, the fused plane pass, finalize); fwd: the plane pass also
// leaves the next step's spectrum.  ev[0..3] bracket the three launches.
// P2 of every member of a group (one launch, grid.y = members)
template <typename T>
void launch_group_pencil(const Instance &L, const Group &G, cudaStream_t st) {
  constexpr int NC = Threads<T>::pencil;
  const unsigned B = (unsigned)G.members.size();
  const InstPtrs *tab = static_cast<const InstPtrs *>(G.table.p);
  PencilArgs pe;
  group_pencil_args<T>(L, pe);
  with_pencil_sc(L.S, [&](auto SCc) {
    k_xpencil_tab<T, NC, decltype(SCc)::value><<<dim3(L.ntiles, B), NC, L.smem_pencil, st>>>(tab, pe);
  });
}

template <typename T>
void enqueue_group_step(Instance &L, const Group &G, cudaStream_t st, double tol, bool fwd, cudaEvent_t *ev = nullptr) {
  const unsigned B = (unsigned)G.members.size();
  const InstPtrs *tab = static_cast<const InstPtrs *>(G.table.p);
  PlaneArgs pa;
  fill_plane_args<T>(L, pa);
  const int planes = L.F * L.nx;
  if (ev) cudaEventRecord(ev[0], st);
  launch_group_pencil<T>(L, G, st);
  if (ev) cudaEventRecord(ev[1], st);
  UpdateArgs ua;
  group_update_args(L, ua);
  launch_step_tab<T>(L, B, st, tab, pa, ua, fwd);
  if (ev) cudaEventRecord(ev[2], st);
  const bool nyq = L.imag == IMAG_NYQ;
  k_finalize_tab<<<B, 1024, 0, st>>>(tab, L.split ? 2 * planes : planes, nyq ? L.ntiles : 0, 1.0 / (double)L.N,
                                     tol);
  if (ev) cudaEventRecord(ev[3], st);
}

// One step of a merge class: three launches for all of its groups.
template <typename T>
void enqueue_merge_step(pfdd_gpu *h, const MergeClass &mc, cudaStream_t st, double tol, bool fwd,
                        cudaEvent_t *ev = nullptr) {
  constexpr int NC = Threads<T>::pencil;
  const Instance &L = *h->inst[h->groups[mc.groups[0]].members[0]];
  if (ev) cudaEventRecord(ev[0], st);
  with_pencil_sc(mc.S, [&](auto SCc) {
    k_xpencil_multi<T, NC, decltype(SCc)::value><<<mc.pencil_ctas, NC, mc.smem_pencil, st>>>(
        mc.pentab.as<MultiPencilGroup>(), mc.mpe, green_host<T>(L.green));
  });
  if (ev) cudaEventRecord(ev[1], st);
  k_step_planes_multi<T, 256><<<mc.plane_ctas, 256, mc.smem_plane, st>>>(mc.ptab.as<MultiPlaneGroup>(), mc.mp,
                                                                         (int)fwd);
  if (ev) cudaEventRecord(ev[2], st);
  k_finalize_multi<<<mc.insts, 1024, 0, st>>>(mc.ftab.as<MultiFinalGroup>(), mc.mf, tol);
  if (ev) cudaEventRecord(ev[3], st);
}

template <typename T>
void enqueue_open_all(pfdd_gpu *h, cudaStream_t st) {
  for (size_t gi = 0; gi < h->groups.size(); ++gi)
    if (h->group_merge[gi] < 0) enqueue_group_open<T>(*h->inst[h->groups[gi].members[0]], h->groups[gi], st);
  for (auto &mc : h->merges)
    k_fwd_planes_multi<T, 256><<<mc.plane_ctas, 256, mc.smem_plane, st>>>(mc.ptab.as<MultiPlaneGroup>(), mc.mp);
}

// Launch units of one step: merge classes and groups outside them.
inline int n_units(const pfdd_gpu *h) {
  int n = (int)h->merges.size();
  for (int m : h->group_merge) n += m < 0;
  return n;
}

// ev: 4 events per unit (n_units of them), in unit order
template <typename T>
void enqueue_all_groups(pfdd_gpu *h, cudaStream_t st, double tol, bool fwd, cudaEvent_t *ev = nullptr) {
  for (size_t gi = 0; gi < h->groups.size(); ++gi)
    if (h->group_merge[gi] < 0) {
      enqueue_group_step<T>(*h->inst[h->groups[gi].members[0]], h->groups[gi], st, tol, fwd, ev);
      if (ev) ev += 4;
    }
  for (auto &mc : h->merges) {
    enqueue_merge_step<T>(h, mc, st, tol, fwd, ev);
    if (ev) ev += 4;
  }
}

constexpr int kLaunchesPerStep = 3;   // per group, plus one opening P1 per run

pfdd_status ensure_stats(pfdd_gpu *h, int cap);
pfdd_status reset_counters(pfdd_gpu *h);
pfdd_status collect(pfdd_gpu *h, pfdd_step_stats *stats);
template <typename T> void stress_all(pfdd_gpu *h, int mode);

template <typename T>
pfdd_status profile_impl(pfdd_gpu *h, int n_steps, double *kernel_ms) {
  cudaStream_t st = h->stream;
  for (int k = 0; k < PFDD_NKERNELS; ++k) kernel_ms[k] = 0.0;
  pfdd_status ps;
  if ((ps = ensure_stats(h, n_steps))) return ps;
  if ((ps = reset_counters(h))) return ps;
  stress_all<T>(h, 0);
  const size_t ng = (size_t)n_units(h);
  std::vector<cudaEvent_t> ev(4 * (size_t)n_steps * ng + 2);
  for (auto &e : ev) CUDA_TRY(h, cudaEventCreate(&e));
  cudaEventRecord(ev[0], st);
  enqueue_open_all<T>(h, st);
  cudaEventRecord(ev[1], st);
  size_t q = 2;
  for (int it = 0; it < n_steps; ++it) {
    enqueue_all_groups<T>(h, st, 0.0, it + 1 < n_steps, &ev[q]);
    q += 4 * ng;
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    kernel_ms[PFDD_K_FWD_PLANES] = ms;
    for (size_t b = 2; b < q; b += 4)
      for (int k = 0; k < 3; ++k) {
        ms = 0.f;
        cudaEventElapsedTime(&ms, ev[b + k], ev[b + k + 1]);
        kernel_ms[PFDD_K_XPENCIL + k] += ms;
      }
    for (int k = 0; k < PFDD_NKERNELS; ++k) kernel_ms[k] /= (double)n_steps;
  }
  for (auto &x : ev) cudaEventDestroy(x);
  CUDA_TRY(h, e);
  return collect(h, nullptr);
}

// ------------------------------------------------------------ energy
// ------------------------------------------------------------ strain / stress
// The strain and stress diagnostics of the current state (see the header):
// forward planes of xi, the strain pencil pass (six symmetric components),
// the inverse planes of those six fields, then the pointwise stress.  The
// constants follow the reference: Voigt mu and nu for G and the stress
// (fft_fftw_slab.cpp:483-495, 3489-3494), the isotropic compliance S11 = 1/E,
// S12 = -nu/E, S44 = 2 (S11 - S12) (material.cpp:154-156; Voigt E and nu,
// equal to the deck's for the isotropic C the material builds), sigma_rot as
// rotate_stress, <eps0> from the per-system means of Re xi (stressfree_strain).
template <typename T>
pfdd_status strain_stress_impl(pfdd_gpu *h, Instance &I, double *eps, double *sigma, double *ave_eps,
                               double *ave_sigma) {
  using C = cx<T>;
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half;
  cudaStream_t st = h->stream;
  ARM_FLAGS(h, I);
  const size_t N = I.N;
  const int S = I.S;
  // sigma_rot (rotate_stress, fft_fftw_slab.cpp:242-274) of the stress state
  // the current xi was stepped with: the reference outputs inside its GL loop,
  // before sigma += dsigma (solve_GL.cpp:110-155), while pfdd_gpu_advance has
  // already added the increment when it returns
  double sig[9], sr[3][3];
  const int nb = 4 * h->nsm;   // reduction blocks of the field sums
  DevBuf &part = I.ss_part, &spec6 = I.ss_spec6, &strain6 = I.ss_strain6, &e9 = I.ss_e9, &s9 = I.ss_s9,
         &fpart = I.ss_fpart;
  const size_t ncols = (size_t)I.ny * I.nzp;
  CUDA_TRY(h, grow(st, part, (size_t)nb * S * sizeof(double)));
  CUDA_TRY(h, grow(st, spec6, 6 * (size_t)I.nx * ncols * sizeof(C)));
  CUDA_TRY(h, grow(st, strain6, 6 * N * sizeof(T)));
  CUDA_TRY(h, grow(st, fpart, (size_t)nb * 18 * sizeof(double)));
  if (eps) CUDA_TRY(h, grow(st, e9, 9 * N * sizeof(double)));
  if (sigma) CUDA_TRY(h, grow(st, s9, 9 * N * sizeof(double)));
  CUDA_TRY(h, cudaMemcpyAsync(sig, I.sigma(), sizeof sig, cudaMemcpyDeviceToHost, st));

  // forward planes of the current state into the spectrum buffer
  PlaneArgs pa;
  fill_plane_args<T>(I, pa);
  launch_fwd<T>(I, st, I.xi[I.cur].as<T>(), I.spec.as<C>(), pa, nullptr, I.flags() + 3);
  const double C44 = I.d.C44, C12 = I.d.C12, C11 = I.d.C11;
  const double mu = C44 - (2.0 * C44 + C12 - C11) / 5.0, ll = C12 - (2.0 * C44 + C12 - C11) / 5.0;
  // strain pencils: tile width reduced until max(F, 6) fields fit
  const int FB = std::max(I.F, 6);
  int cc = I.ccols;
  // field stride padded against bank conflicts, as the x-pencil pass's
  auto bytes = [&](int c) { return ((size_t)FB * pencil_fstride<T>(I, c) + I.nx) * sizeof(C); };
  while (cc > 1 && bytes(cc) > 227 * 1024) cc >>= 1;
  if (bytes(cc) > 227 * 1024 || ncols % cc)
    return fail(h, PFDD_EUNSUPPORTED, "strain pencil of %d x %d fields does not fit shared memory", I.nx, FB);
  CUDA_TRY(h, raise_smem_limit(k_strain_pencil<T, 256>, bytes(cc)));
  PencilArgs pe{};
  pe.px = I.px;
  pe.nx = I.nx; pe.ny = I.ny; pe.nz = I.nz; pe.nzh = I.nzh; pe.nzp = I.nzp; pe.M = I.M;
  pe.S = I.S; pe.F = I.F; pe.imag = I.imag;
  pe.ncols = (int)ncols;
  pe.ccols = cc;
  pe.tw_x = I.tw_x.p;
  pe.kx_of = I.kx_of; pe.ky_of = I.ky_of; pe.kz_of = I.kz_of;
  pe.mode = PASS_STEP;
  pe.fstride = pencil_fstride<T>(I, cc);
  pe.aux = I.aux.p;
  pe.sx_n = I.sx_n; pe.sy_n = I.sy_n;
  pe.g = I.green;
  set_pencil_divisors<T>(pe);
  pe.fd_6cc = FastDiv(6 * cc);
  pe.inv2mu = 0.5 / mu;
  k_strain_pencil<T, 256><<<(unsigned)(ncols / cc), 256, bytes(cc), st>>>(I.spec.as<C>(), spec6.as<C>(), pe);
  // inverse planes of the six strain spectra (the Im-synthesis pass: IFFT / N)
  {
    UpdateArgs ua;
    memset(&ua, 0, sizeof ua);
    ua.nx = I.nx; ua.ny = I.ny; ua.nz = I.nz; ua.nzh = I.nzh; ua.nzp = I.nzp; ua.S = I.S; ua.F = 6;
    ua.invN = 1.0 / (double)N;
    ua.core = I.core;
    ua.err = I.flags() + 3;
    ua.mode = PASS_SYNTH;
    const unsigned planes6 = (unsigned)(6 * I.nx);
    if (I.split)
      launch_pair(k_inv_update<T, NH, true>, dim3(2 * planes6), NH, I.smem_update, st, spec6.as<C>(),
                  I.xi[I.cur].as<T>(), strain6.as<T>(), pa, ua, I.partials.as<double>());
    else
      k_inv_update<T, NP, false><<<planes6, NP, I.smem_update, st>>>(spec6.as<C>(), I.xi[I.cur].as<T>(),
                                                                       strain6.as<T>(), pa, ua,
                                                                       I.partials.as<double>());
  }
  // per-system sums of Re xi of the current state, read back once the
  // transforms are queued (the host forms the stress constants from them)
  k_field_sums<T><<<nb, 256, 0, st>>>(I.xi[I.cur].as<T>(), S, N, part.as<double>());
  // averages only: the six strain sums are all the device still has to add
  // (the stress average is linear in them and in the sums of Re xi above)
  const bool ave_only = !eps && !sigma;
  if (ave_only) k_field_sums<T><<<nb, 256, 0, st>>>(strain6.as<T>(), 6, N, fpart.as<double>());
  std::vector<double> hp((size_t)nb * S), h6(ave_only ? (size_t)nb * 6 : 0);
  CUDA_TRY(h, cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (ave_only)
    CUDA_TRY(h, cudaMemcpyAsync(h6.data(), fpart.p, h6.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  const StressArgs &sa = I.stress;
  if (I.advanced)
    for (int i = 0; i < 9; ++i) sig[i] -= I.d.dsigma[i / 3][i % 3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      if (sa.ortho) {
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) v += sa.prim[i][k] * sig[3 * k + l] * sa.invprim[l][j];
      } else {
        v = sig[3 * i + j];
      }
      sr[i][j] = v;
    }
  const double young = mu * (3 * ll + 2 * mu) / (ll + mu), xnu = young / 2.0 / mu - 1.0;
  const double S11 = 1.0 / young, S12 = -xnu / young, S44 = 2.0 * (S11 - S12);
  double epsm[PFDD_MAXS][3][3], mean[PFDD_MAXS];
  for (int a = 0; a < S; ++a) {
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += hp[(size_t)b * S + a];
    mean[a] = t / (double)N;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) epsm[a][i][j] = I.d.xb[a][i] * I.d.xn[a][j] / I.d.dslip;
  }
  double avepsts[3][3], avepst[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) {
          const double Sijkl = S44 / 4.0 * ((i == k && j == l) + (i == l && j == k)) + S12 * (i == j && k == l);
          v += Sijkl * sr[k][l] * mu;
        }
      avepsts[i][j] = v;
      double e0 = 0.0;
      for (int a = 0; a < S; ++a) e0 += epsm[a][i][j] * mean[a];
      avepst[i][j] = v + e0;
    }
  StressFieldArgs sp;
  memset(&sp, 0, sizeof sp);
  const int qi[6] = {0, 1, 2, 0, 0, 1}, qj[6] = {0, 1, 2, 1, 2, 2};
  for (int q = 0; q < 6; ++q) {
    const int i = qi[q], j = qj[q];
    for (int a = 0; a < S; ++a) sp.e6[a][q] = 0.5 * (epsm[a][i][j] + epsm[a][j][i]);
    sp.avepst6[q] = 0.5 * (avepst[i][j] + avepst[j][i]);
    sp.avepsts6[q] = 0.5 * (avepsts[i][j] + avepsts[j][i]);
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) sp.sigmu[3 * i + j] = sr[i][j] * mu;
  sp.C44 = C44;
  sp.C12 = C12;
  sp.S = S;

  auto neumaier = [](const double *v, int n, int stride) {
    double t = 0.0, c = 0.0;
    for (int b = 0; b < n; ++b) {
      const double x = v[(size_t)b * stride], u = t + x;
      c += (std::fabs(t) >= std::fabs(x)) ? (t - u) + x : (x - u) + t;
      t = u;
    }
    return t + c;
  };
  if (ave_only) {
    // <eps_q> = <strain_q> + avepst_q; <X_q> = <eps_q> - sum_s e6[s][q] <Re xi_s> - avepsts_q;
    // <sigma_ij> = 2 C44 <X_q> + C12 tr<X> delta_ij + sigma_rot mu (k_stress_fields, averaged)
    int fl[4];
    CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
    if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
    double em[6], xm[6];
    for (int q = 0; q < 6; ++q) {
      em[q] = neumaier(h6.data() + q, nb, 6) / (double)N + sp.avepst6[q];
      double d = 0.0;
      for (int a = 0; a < S; ++a) d += sp.e6[a][q] * mean[a];
      xm[q] = em[q] - d - sp.avepsts6[q];
    }
    const int map[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
    const double tr = xm[0] + xm[1] + xm[2];
    for (int ij = 0; ij < 9; ++ij) {
      const int i = ij / 3, j = ij - 3 * i, q = map[ij];
      if (ave_eps) ave_eps[ij] = em[q];
      if (ave_sigma) ave_sigma[ij] = 2.0 * C44 * xm[q] + (i == j ? C12 * tr : 0.0) + sp.sigmu[ij];
    }
    return PFDD_OK;
  }

  // pointwise strain and stress, FP64 sums of both
  k_stress_fields<T><<<nb, 256, 0, st>>>(strain6.as<T>(), I.xi[I.cur].as<T>(), N, sp,
                                          eps ? e9.as<double>() : nullptr, sigma ? s9.as<double>() : nullptr,
                                          fpart.as<double>());
  std::vector<double> hf((size_t)nb * 18);
  CUDA_TRY(h, cudaMemcpyAsync(hf.data(), fpart.p, hf.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (eps) CUDA_TRY(h, cudaMemcpyAsync(eps, e9.p, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (sigma) CUDA_TRY(h, cudaMemcpyAsync(sigma, s9.p, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  int fl[4];
  CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
  if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
  for (int q = 0; q < 18; ++q) {
    const double m = neumaier(hf.data() + q, nb, 18) / (double)N;   // Neumaier-compensated
    if (q < 9 && ave_eps) ave_eps[q] = m;
    if (q >= 9 && ave_sigma) ave_sigma[q - 9] = m;
  }
  return PFDD_OK;
}

// E_elastic = 1/2 <xi, L xi> (Re and Im), E_core = sum f(Re xi),
// E_applied = -sum tau_a Re xi_a, from one elastic pass of the current state.
template <typename T>
pfdd_status energy_impl(pfdd_gpu *h, Instance &I, double *e_el, double *e_core, double *e_app) {
  cudaStream_t st = h->stream;
  ARM_FLAGS(h, I);
  DevBuf gpart;
  CUDA_TRY(h, gpart.alloc(4 * (size_t)I.F * I.nx * sizeof(double)));
  k_stress_state<<<1, 32, 0, st>>>(I.sigma(), I.tau(), I.an(), I.stress, 0, nullptr);
  PlaneArgs pa;
  fill_plane_args<T>(I, pa);
  const T *xcur = I.xi[I.cur].as<T>();
  cx<T> *spec = I.spec.as<cx<T>>();
  const int planes = I.F * I.nx;
  launch_fwd<T>(I, st, xcur, spec, pa, nullptr, I.flags() + 3);
  PencilArgs pe;
  pe = PencilArgs{};
  pe.px = I.px;
  pe.nx = I.nx; pe.ny = I.ny; pe.nz = I.nz; pe.nzh = I.nzh; pe.nzp = I.nzp; pe.M = I.M;
  pe.S = I.S; pe.F = I.F; pe.imag = I.imag;
  pe.ncols = I.ny * I.nzp;
  pe.ccols = I.ccols;
  pe.tw_x = I.tw_x.p;
  pe.kx_of = I.kx_of; pe.ky_of = I.ky_of; pe.kz_of = I.kz_of;
  pe.mode = PASS_ENERGY;
  pe.fstride = I.fstride;
  pe.aux = I.aux.p;
  pe.sx_n = I.sx_n; pe.sy_n = I.sy_n;
  pe.cd = I.d.cd_dt;
  pe.partials = I.imag == IMAG_NYQ ? I.ppart.as<double>() : nullptr;
  pe.g = I.green;
  set_pencil_divisors<T>(pe);
  launch_pencil<T>(I, st, spec, pe, nullptr);
  UpdateArgs ua;
  memset(&ua, 0, sizeof ua);
  ua.nx = I.nx; ua.ny = I.ny; ua.nz = I.nz; ua.nzh = I.nzh; ua.nzp = I.nzp; ua.S = I.S; ua.F = I.F;
  ua.cd = I.d.cd_dt;
  ua.invN = 1.0 / (double)I.N;
  ua.core = I.core;
  ua.tau = I.tau();
  ua.mask = I.mask.as<uint8_t>();
  ua.site = I.site_arg;
  ua.err = I.flags() + 3;
  ua.mode = PASS_ENERGY;
  ua.gpart = gpart.as<double>();
  // xout is not written by the energy pass
  launch_inv<T>(I, planes, st, spec, xcur, I.xi[I.cur ^ 1].as<T>(), pa, ua,
                                                        I.partials.as<double>());
  std::vector<double> gp(4 * (size_t)planes), pp;
  CUDA_TRY(h, cudaMemcpyAsync(gp.data(), gpart.p, gp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (I.imag == IMAG_NYQ) {
    pp.resize(2 * (size_t)I.ntiles);
    CUDA_TRY(h, cudaMemcpyAsync(pp.data(), I.ppart.p, pp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(h, cudaStreamSynchronize(st));
  CUDA_TRY(h, cudaGetLastError());
  {
    int fl[4];
    CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
    if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
  }
  // compensated (Neumaier) sums in FP64
  auto sum = [](const double *v, size_t n, size_t stride, double scale) {
    double s = 0.0, c = 0.0;
    for (size_t i = 0; i < n; ++i) {
      const double x = v[i * stride] * scale, t = s + x;
      c += (std::fabs(s) >= std::fabs(x)) ? (s - t) + x : (x - t) + s;
      s = t;
    }
    return s + c;
  };
  double el = sum(gp.data(), planes, 4, 1.0);
  if (!pp.empty()) el += sum(pp.data(), I.ntiles, 2, 1.0 / (double)I.N);
  if (e_el) *e_el = el;
  if (e_core) *e_core = sum(gp.data() + 1, planes, 4, 1.0);
  if (e_app) *e_app = sum(gp.data() + 2, planes, 4, 1.0);
  return PFDD_OK;
}

// ------------------------------------------------------------ adjoint
// Reverse-mode gradient of a loss L(Re xi_N), xi_N = n_steps GL iterations
// from the current state at the current stress state, in two calls:
//   adjoint_forward_impl  the forward run, kept as a tape: the state every K
//                         steps (with the Nyquist carrier of Im xi), and every
//                         state of the last segment; the instance ends at xi_N;
//   adjoint_backward_impl seeded with dL/dRe xi_N, each segment's states
//                         recomputed from its checkpoint (the last segment's
//                         are on the tape already), then the adjoint steps
//   lam_n = lam_{n+1} - cd (L lam_{n+1} + f''(xi_n) lam_{n+1}),
// whose plane passes add their per-plane gradient sums into one accumulator;
// one reduction at the end.  The tape stays valid (several seeds may be
// run) until the instance's state changes.  Tape steps leave out the per-step
// reduction (no xinorm is needed); a non-finite gradient reports divergence.
template <typename T>
pfdd_status adjoint_forward_impl(pfdd_gpu *h, Instance &I, int n_steps, int K) {
  cudaStream_t st = h->stream;
  ARM_FLAGS(h, I);
  I.tape_steps = 0;
  const size_t n_all = (size_t)I.F * I.N, sb = n_all * sizeof(T);
  const size_t aux_bytes = I.aux.bytes;
  const int nck = (n_steps + K - 1) / K;
  const int last0 = (nck - 1) * K;            // first step of the last segment
  const int seg_slots = n_steps - last0;      // states n = last0 .. n_steps-1
  auto need = [&](DevBuf &b, size_t bytes) -> cudaError_t {
    if (b.bytes >= bytes && b.p) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    b.release();
    return b.alloc(bytes);
  };
  // the last segment's states stay on the tape (adj_last); earlier segments
  // are recomputed into adj_seg[j & 1] during the backward pass
  CUDA_TRY(h, need(I.adj_ck, (size_t)nck * (sb + aux_bytes)));
  CUDA_TRY(h, need(I.adj_last, (size_t)seg_slots * sb));
  for (int b = 0; b < std::min(2, nck - 1); ++b) CUDA_TRY(h, need(I.adj_seg[b], (size_t)K * sb));
  CUDA_TRY(h, need(I.adj_fin, sb));
  if (aux_bytes) CUDA_TRY(h, need(I.adj_finaux, aux_bytes));
  auto ck_state = [&](int j) { return I.adj_ck.as<char>() + (size_t)j * (sb + aux_bytes); };
  auto slot = [&](int n) { return I.adj_last.as<char>() + (size_t)(n - last0) * sb; };
  k_stress_state<<<1, 32, 0, st>>>(I.sigma(), I.tau(), I.an(), I.stress, 0, I.flags());
  PlaneArgs pa;
  fill_plane_args<T>(I, pa);
  // the opening transform, then fused steps; state n lives in I.xi (n < last0)
  // or in its tape slot (n >= last0)
  const void *cur = I.xi[I.cur].p;
  launch_fwd<T>(I, st, static_cast<const T *>(cur), I.spec.as<cx<T>>(), pa, I.flags(), I.flags() + 3);
  int pp = I.cur;   // ping-pong index of the state in I.xi while n < last0
  for (int n = 0; n < n_steps; ++n) {
    if (n % K == 0) {
      CUDA_TRY(h, cudaMemcpyAsync(ck_state(n / K), cur, sb, cudaMemcpyDeviceToDevice, st));
      if (aux_bytes)
        CUDA_TRY(h, cudaMemcpyAsync(ck_state(n / K) + sb, I.aux.p, aux_bytes, cudaMemcpyDeviceToDevice, st));
    }
    if (n == last0 && cur != slot(n)) {   // the last segment's first state onto the tape
      CUDA_TRY(h, cudaMemcpyAsync(slot(n), cur, sb, cudaMemcpyDeviceToDevice, st));
      cur = slot(n);
    }
    void *out;
    if (n + 1 == n_steps) out = I.xi[I.cur ^ 1].p;      // xi_N where the instance keeps its state
    else if (n + 1 >= last0) out = slot(n + 1);
    else {
      pp ^= 1;
      out = I.xi[pp].p;
    }
    enqueue_step_fused<T>(I, st, n + 1 < n_steps, nullptr, cur, out, false);
    cur = out;
  }
  I.cur ^= 1;
  CUDA_TRY(h, cudaMemcpyAsync(I.flags() + 4, &I.cur, sizeof(int), cudaMemcpyHostToDevice, st));
  // xi_N and its carrier, restored after the backward pass reuses the buffers
  CUDA_TRY(h, cudaMemcpyAsync(I.adj_fin.p, I.xi[I.cur].p, sb, cudaMemcpyDeviceToDevice, st));
  if (aux_bytes) CUDA_TRY(h, cudaMemcpyAsync(I.adj_finaux.p, I.aux.p, aux_bytes, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  CUDA_TRY(h, cudaGetLastError());
  int fl[4];
  CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
  if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
  I.tape_steps = n_steps;
  I.tape_K = K;
  return PFDD_OK;
}

template <typename T>
pfdd_status adjoint_backward_impl(pfdd_gpu *h, Instance &I, const double *seed, double *dparams, double *dsigma) {
  cudaStream_t st = h->stream;
  if (I.tape_steps < 1) return fail(h, PFDD_ESTATE, "no adjoint tape: call pfdd_gpu_adjoint_forward first");
  ARM_FLAGS(h, I);
  const int n_steps = I.tape_steps, K = I.tape_K;
  const size_t n_re = (size_t)I.S * I.N, n_all = (size_t)I.F * I.N, sb = n_all * sizeof(T);
  const size_t aux_bytes = I.aux.bytes;
  const int nck = (n_steps + K - 1) / K;
  auto need = [&](DevBuf &b, size_t bytes) -> cudaError_t {
    if (b.bytes >= bytes && b.p) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    b.release();
    return b.alloc(bytes);
  };
  DevBuf *lam = I.adj_lam;
  for (int b = 0; b < 2; ++b) CUDA_TRY(h, need(lam[b], sb));
  if (aux_bytes) CUDA_TRY(h, need(I.adj_aux, aux_bytes));
  CUDA_TRY(h, need(I.adj_gpart, 4 * (size_t)I.F * I.nx * sizeof(double)));
  CUDA_TRY(h, need(I.adj_acc, 2 * (2 + PFDD_MAXS) * sizeof(double)));
  CUDA_TRY(h, cudaMemsetAsync(I.adj_acc.p, 0, I.adj_acc.bytes, st));
  CUDA_TRY(h, cudaMemsetAsync(I.adj_gpart.p, 0, I.adj_gpart.bytes, st));
  // seed: lam_N = dL/dRe xi_N on the real fields, 0 on Im (and its carrier)
  if (h->staging.bytes < 2 * n_re * sizeof(double)) {
    CUDA_TRY(h, cudaStreamSynchronize(st));
    h->staging.release();
    CUDA_TRY(h, h->staging.alloc(2 * n_re * sizeof(double)));
  }
  CUDA_TRY(h, cudaMemcpyAsync(h->staging.p, seed, n_re * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(h, cudaMemsetAsync(lam[0].p, 0, sb, st));
  k_from_planar<T><<<1184, 256, 0, st>>>(h->staging.as<double>(), lam[0].as<T>(), n_re);
  if (aux_bytes) CUDA_TRY(h, cudaMemsetAsync(I.adj_aux.p, 0, aux_bytes, st));
  auto ck_state = [&](int j) { return I.adj_ck.as<char>() + (size_t)j * (sb + aux_bytes); };
  k_stress_state<<<1, 32, 0, st>>>(I.sigma(), I.tau(), I.an(), I.stress, 0, I.flags());
  PlaneArgs pa;
  fill_plane_args<T>(I, pa);
  // Segment j - 1 is recomputed on a second stream while segment j runs
  // backwards (the two chains share no buffer: the recomputation has its own
  // spectrum, carrier and one of two state buffers), so small grids keep the
  // SMs busy with two independent chains.
  if (nck > 1) {
    CUDA_TRY(h, need(I.adj_rspec, I.spec.bytes));
    if (aux_bytes) CUDA_TRY(h, need(I.adj_raux, aux_bytes));
    if (!h->side_stream) CUDA_TRY(h, cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking));
  }
  cudaStream_t rs = h->side_stream;
  std::vector<cudaEvent_t> evs;
  auto event = [&](cudaEvent_t *e) -> cudaError_t {
    cudaError_t r = cudaEventCreateWithFlags(e, cudaEventDisableTiming);
    if (r == cudaSuccess) evs.push_back(*e);
    return r;
  };
  struct EvGuard {
    std::vector<cudaEvent_t> &v;
    ~EvGuard() {
      for (auto e : v) cudaEventDestroy(e);
    }
  } guard{evs};
  std::vector<cudaEvent_t> rec_done(nck, nullptr), bwd_done(nck, nullptr);
  auto seg_states = [&](int j) { return (j == nck - 1 ? I.adj_last : I.adj_seg[j & 1]).as<char>(); };
  // recompute segment j's states (from its checkpoint) on the side stream
  auto recompute = [&](int j) -> pfdd_status {
    const int n0 = j * K, n1 = std::min(n_steps, n0 + K);
    char *states = seg_states(j);
    auto slot = [&](int i) { return states + (size_t)i * sb; };
    CUDA_TRY(h, cudaMemcpyAsync(slot(0), ck_state(j), sb, cudaMemcpyDeviceToDevice, rs));
    if (aux_bytes)
      CUDA_TRY(h, cudaMemcpyAsync(I.adj_raux.p, ck_state(j) + sb, aux_bytes, cudaMemcpyDeviceToDevice, rs));
    if (n1 - n0 > 1)
      launch_fwd<T>(I, rs, reinterpret_cast<const T *>(slot(0)), I.adj_rspec.as<cx<T>>(), pa, I.flags(),
                    I.flags() + 3);
    for (int n = n0; n + 1 < n1; ++n)
      enqueue_step_fused<T>(I, rs, n + 2 < n1, nullptr, slot(n - n0), slot(n + 1 - n0), false, I.adj_rspec.p,
                            aux_bytes ? I.adj_raux.p : nullptr);
    CUDA_TRY(h, event(&rec_done[j]));
    CUDA_TRY(h, cudaEventRecord(rec_done[j], rs));
    return PFDD_OK;
  };
  if (nck > 1) {
    cudaEvent_t start;
    CUDA_TRY(h, event(&start));
    CUDA_TRY(h, cudaEventRecord(start, st));   // tau and flags are set
    CUDA_TRY(h, cudaStreamWaitEvent(rs, start, 0));
    pfdd_status ps = recompute(nck - 2);
    if (ps != PFDD_OK) return ps;
  }
  int lc = 0;
  for (int j = nck - 1; j >= 0; --j) {
    const int n0 = j * K, n1 = std::min(n_steps, n0 + K);
    // the next segment down is recomputed beside this one's backward steps,
    // into the state buffer the segment above used (free once it is done)
    if (j - 1 >= 0 && j - 1 != nck - 2) {
      if (j + 1 <= nck - 2) CUDA_TRY(h, cudaStreamWaitEvent(rs, bwd_done[j + 1], 0));
      pfdd_status ps = recompute(j - 1);
      if (ps != PFDD_OK) return ps;
    }
    if (j != nck - 1) CUDA_TRY(h, cudaStreamWaitEvent(st, rec_done[j], 0));
    char *states = seg_states(j);
    auto slot = [&](int i) { return states + (size_t)i * sb; };
    // backward steps: each plane pass also transforms the new lambda
    launch_fwd<T>(I, st, lam[lc].as<T>(), I.spec.as<cx<T>>(), pa, I.flags(), I.flags() + 3);
    for (int n = n1 - 1; n >= n0; --n) {
      AdjointPass ap{lam[lc].p, lam[lc ^ 1].p, slot(n - n0), I.adj_aux.p, I.adj_gpart.as<double>()};
      enqueue_step_fused<T>(I, st, n > n0, &ap);
      lc ^= 1;
    }
    CUDA_TRY(h, event(&bwd_done[j]));
    CUDA_TRY(h, cudaEventRecord(bwd_done[j], st));
  }
  k_grad_accum<<<1, 32, 0, st>>>(I.adj_gpart.as<double>(), I.S, I.nx, I.adj_acc.as<double>(),
                                  I.adj_acc.as<double>() + 2 + PFDD_MAXS);
  // hand back xi_N (the recomputation reused the carrier)
  CUDA_TRY(h, cudaMemcpyAsync(I.xi[I.cur].p, I.adj_fin.p, sb, cudaMemcpyDeviceToDevice, st));
  if (aux_bytes) CUDA_TRY(h, cudaMemcpyAsync(I.aux.p, I.adj_finaux.p, aux_bytes, cudaMemcpyDeviceToDevice, st));
  double hacc[2 * (2 + PFDD_MAXS)];
  CUDA_TRY(h, cudaMemcpyAsync(hacc, I.adj_acc.p, sizeof hacc, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  CUDA_TRY(h, cudaGetLastError());
  int fl[4];
  CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
  if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
  const double cd = I.d.cd_dt;
  double A[2 + PFDD_MAXS];
  for (int t = 0; t < 2 + I.S; ++t) {
    A[t] = hacc[t] + hacc[2 + PFDD_MAXS + t];
    if (!std::isfinite(A[t])) return fail(h, PFDD_EDIVERGED, "non-finite adjoint sums");
  }
  if (dparams) {
    dparams[0] = -cd * A[0];
    dparams[1] = -cd * A[1];
  }
  if (dsigma) {
    // dJ/dtau_a = cd * sum lambda_a; tau_a = sum_ij sigma_rot_ij P_a,ij / dslip with
    // P_a,ij = xb_ai xn_aj (Schmid) or S_tot (non-Schmid).  Core model 6 adds
    // dJ/dAn dAn/dsigma_rot[2][1], An = 1e-3 gsfe(sigma_rot[2][1]).
    const StressArgs &sa = I.stress;
    const double dAn_dsr21 =
        sa.usfe ? 1.0E-3 * (sa.fit[0] * sa.mu * 1.0E-9 * sa.fit_sin + sa.fit[3] * sa.mu * 1.0E-9) : 0.0;
    const double dJ_dAn = -cd * A[0];
    const int comp[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int c = 0; c < 6; ++c) {
      double g = 0.0;
      for (int a = 0; a < I.S; ++a) {
        double dt = 0.0;
        for (int pass = 0; pass < (comp[c][0] == comp[c][1] ? 1 : 2); ++pass) {
          const int k = pass ? comp[c][1] : comp[c][0], l = pass ? comp[c][0] : comp[c][1];
          for (int i = 0; i < 3; ++i)
            for (int jj = 0; jj < 3; ++jj) {
              const double dr = sa.ortho ? sa.prim[i][k] * sa.invprim[l][jj] : ((i == k && jj == l) ? 1.0 : 0.0);
              dt += dr * (sa.ns ? sa.proj[a][i][jj] : sa.xn[a][jj] * sa.xb[a][i]) / sa.dslip;
            }
        }
        g += cd * A[2 + a] * dt;
      }
      if (sa.usfe) {
        double d21 = 0.0;
        for (int pass = 0; pass < (comp[c][0] == comp[c][1] ? 1 : 2); ++pass) {
          const int k = pass ? comp[c][1] : comp[c][0], l = pass ? comp[c][0] : comp[c][1];
          d21 += sa.ortho ? sa.prim[2][k] * sa.invprim[l][1] : ((k == 2 && l == 1) ? 1.0 : 0.0);
        }
        g += dJ_dAn * dAn_dsr21 * d21;
      }
      dsigma[c] = g;
    }
  }
  return PFDD_OK;
}

// Graph of `steps` GL iterations of every group (states = 0), or of `states`
// whole stress states of `steps` iterations each (tau from sigma, the steps,
// sigma += dsigma), captured once per key.  One opening forward pass, then
// every plane pass but the last leaves the next step's spectrum: the forward
// spectrum does not depend on the stress, and an instance that stopped on
// the tolerance keeps the spectrum of its current state.
template <typename T>
pfdd_status graph_for(pfdd_gpu *h, int steps, int states, double tol, cudaGraphExec_t *out) {
  GraphKey key{steps, states, tol};
  auto it = h->graphs.find(key);
  if (it != h->graphs.end()) { *out = it->second; return PFDD_OK; }
  cudaStream_t st = h->stream;
  cudaGraph_t g;
  CUDA_TRY(h, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  if (states == 0) {
    enqueue_open_all<T>(h, st);
    for (int i = 0; i < steps; ++i) enqueue_all_groups<T>(h, st, tol, i + 1 < steps);
  } else {
    for (int j = 0; j < states; ++j) {
      stress_all<T>(h, 0);   // clears the stop flags before the opening pass reads them
      if (j == 0) enqueue_open_all<T>(h, st);
      for (int i = 0; i < steps; ++i)
        enqueue_all_groups<T>(h, st, tol, !(j + 1 == states && i + 1 == steps));
      stress_all<T>(h, 1);
    }
  }
  CUDA_TRY(h, cudaStreamEndCapture(st, &g));
  cudaGraphExec_t ge;
  cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  CUDA_TRY(h, e);
  h->graphs[key] = ge;
  *out = ge;
  return PFDD_OK;
}

// Grow every instance's per-step record buffer to `cap` records.
pfdd_status ensure_stats(pfdd_gpu *h, int cap) {
  bool changed = false;
  for (auto &ip : h->inst) {
    Instance &I = *ip;
    if (I.stats_cap >= cap) continue;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    I.stats.release();
    CUDA_TRY(h, I.stats.alloc(2 * (size_t)cap * sizeof(double)));
    I.stats_cap = cap;
    changed = true;
  }
  return changed ? refresh_tables(h) : PFDD_OK;
}

// Read back each instance's control words after a run; keeps the host mirror
// of the current buffer in step with the device.
pfdd_status collect(pfdd_gpu *h, pfdd_step_stats *stats) {
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < h->inst.size(); ++i) {
    Instance &I = *h->inst[i];
    int fl[5];
    CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
    I.cur = fl[4];   // the device's buffer selector, also after an error
    if (fl[3]) return fail(h, PFDD_ETIMEOUT, "instance %zu: a bounded device wait ran out", i);
    if (fl[1]) return fail(h, PFDD_EDIVERGED, "instance %zu: non-finite order parameter", i);
    const int did = std::min(fl[2], I.stats_cap);
    I.hist.resize(2 * (size_t)did);
    if (did)
      CUDA_TRY(h, cudaMemcpy(I.hist.data(), I.stats.p, 2 * (size_t)did * sizeof(double), cudaMemcpyDeviceToHost));
    I.hist_count = did;
    I.steps_total += (unsigned long long)fl[2];
    if (stats) {
      stats[i].steps_done = fl[2];
      stats[i].converged = fl[0];
      stats[i].xinorm = did ? I.hist[2 * (did - 1)] : 0.0;
      stats[i].xiave = did ? I.hist[2 * (did - 1) + 1] : 0.0;
    }
  }
  return PFDD_OK;
}

pfdd_status reset_counters(pfdd_gpu *h) {
  for (auto &ip : h->inst) {
    ip->tape_steps = 0;   // the state moves on: the adjoint tape no longer describes it
    CUDA_TRY(h, cudaMemsetAsync(ip->flags() + 2, 0, sizeof(int), h->stream));
    ARM_FLAGS(h, *ip);
  }
  return PFDD_OK;
}

template <typename T>
void stress_all(pfdd_gpu *h, int mode) {
  for (auto &G : h->groups)
    k_stress_state_tab<<<(unsigned)G.members.size(), 32, 0, h->stream>>>(
        static_cast<const InstPtrs *>(G.table.p), h->inst[G.members[0]]->stress, mode);
}

template <typename T>
pfdd_status advance_impl(pfdd_gpu *h, int n_steps, int stress_states, double tol, pfdd_step_stats *stats) {
  cudaStream_t st = h->stream;
  pfdd_status ps;
  const long long total = (long long)n_steps * stress_states;
  if ((ps = ensure_stats(h, (int)std::min<long long>(total, 1 << 24)))) return ps;
  if ((ps = reset_counters(h))) return ps;
  const int chunk = 32;
  if (h->opt.use_graphs && n_steps < chunk && stress_states > 1) {
    // short stress states (a ramp): several whole states per graph
    const int per = chunk / n_steps;
    for (int left = stress_states; left > 0;) {
      const int k = std::min(per, left);
      cudaGraphExec_t ge = nullptr;
      if ((ps = graph_for<T>(h, n_steps, k, tol, &ge))) return ps;
      CUDA_TRY(h, cudaGraphLaunch(ge, st));
      left -= k;
    }
    for (auto &ip : h->inst) ip->advanced = true;
    CUDA_TRY(h, cudaGetLastError());
    return collect(h, stats);
  }
  for (int ss = 0; ss < stress_states; ++ss) {
    stress_all<T>(h, 0);
    if (h->opt.use_graphs) {
      int left = n_steps;
      while (left > 0) {
        const int k = std::min(chunk, left);
        cudaGraphExec_t ge = nullptr;
        if ((ps = graph_for<T>(h, k, 0, tol, &ge))) return ps;
        CUDA_TRY(h, cudaGraphLaunch(ge, st));
        left -= k;
      }
    } else {
      enqueue_open_all<T>(h, st);
      for (int it = 0; it < n_steps; ++it) enqueue_all_groups<T>(h, st, tol, it + 1 < n_steps);
    }
    stress_all<T>(h, 1);
  }
  for (auto &ip : h->inst) ip->advanced = true;
  CUDA_TRY(h, cudaGetLastError());
  return collect(h, stats);
}

template <typename T>
pfdd_status set_state_impl(pfdd_gpu *h, Instance &I, const double *re, const double *im, bool interleaved) {
  const size_t n = (size_t)I.S * I.N;
  I.tape_steps = 0;
  if (h->staging.bytes < 2 * n * sizeof(double)) {
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->staging.release();
    CUDA_TRY(h, h->staging.alloc(2 * n * sizeof(double)));
  }
  DevBuf &tmp = h->staging;
  T *dre = I.xi[I.cur].as<T>();
  T *dim = I.F > I.S ? dre + n : nullptr;
  if (I.imag == IMAG_NYQ) {
    // the Nyquist carrier starts from Im xi = 0 (what every reference initial_sxtal_* sets)
    if (im)
      for (size_t i = 0; i < n; ++i)
        if (im[i] != 0.0)
          return fail(h, PFDD_EINVAL, "nonzero Im xi needs a handle created with PFDD_IMAG_FULL");
    if (interleaved)
      for (size_t i = 0; i < n; ++i)
        if (re[2 * i + 1] != 0.0)
          return fail(h, PFDD_EINVAL, "nonzero Im xi needs a handle created with PFDD_IMAG_FULL");
    CUDA_TRY(h, cudaMemsetAsync(I.aux.p, 0, I.aux.bytes, h->stream));
  }
  if (interleaved) {
    CUDA_TRY(h, cudaMemcpyAsync(tmp.p, re, 2 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_from_interleaved<T><<<1184, 256, 0, h->stream>>>(tmp.as<double>(), dre, dim, n);
  } else {
    CUDA_TRY(h, cudaMemcpyAsync(tmp.p, re, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_from_planar<T><<<1184, 256, 0, h->stream>>>(tmp.as<double>(), dre, n);
    if (dim) {
      if (im) {
        CUDA_TRY(h, cudaMemcpyAsync(tmp.as<double>() + n, im, n * sizeof(double), cudaMemcpyHostToDevice,
                                    h->stream));
        k_from_planar<T><<<1184, 256, 0, h->stream>>>(tmp.as<double>() + n, dim, n);
      } else {
        CUDA_TRY(h, cudaMemsetAsync(dim, 0, n * sizeof(T), h->stream));
      }
    }
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  CUDA_TRY(h, cudaGetLastError());
  return PFDD_OK;
}

// Im xi of a Nyquist-carrier instance into dst [S*N] (compute precision):
// x-inverse of the Nyquist spectrum (k_xpencil PASS_SYNTH), then the plane
// inverse (k_inv_update PASS_SYNTH), through the spectrum buffer.
template <typename T>
void synth_imag(Instance &I, cudaStream_t st, T *dst) {
  PencilArgs pe;
  pe = PencilArgs{};
  pe.px = I.px;
  pe.nx = I.nx; pe.ny = I.ny; pe.nz = I.nz; pe.nzh = I.nzh; pe.nzp = I.nzp; pe.M = I.M;
  pe.S = I.S; pe.F = I.S; pe.imag = IMAG_NYQ;
  pe.ncols = I.ny * I.nzp;
  pe.ccols = I.ccols;
  pe.tw_x = I.tw_x.p;
  pe.kx_of = I.kx_of; pe.ky_of = I.ky_of; pe.kz_of = I.kz_of;
  pe.mode = PASS_SYNTH;
  pe.fstride = I.fstride;
  pe.aux = I.aux.p;
  pe.sx_n = I.sx_n; pe.sy_n = I.sy_n;
  pe.g = I.green;
  cx<T> *spec = I.spec.as<cx<T>>();
  set_pencil_divisors<T>(pe);
  launch_pencil<T>(I, st, spec, pe, nullptr);
  PlaneArgs pa;
  fill_plane_args<T>(I, pa);
  UpdateArgs ua;
  memset(&ua, 0, sizeof ua);
  ua.nx = I.nx; ua.ny = I.ny; ua.nz = I.nz; ua.nzh = I.nzh; ua.nzp = I.nzp; ua.S = I.S; ua.F = I.S;
  ua.invN = 1.0 / (double)I.N;
  ua.mode = PASS_SYNTH;
  ua.err = I.flags() + 3;
  // xin is not read by the synthesis pass
  launch_inv<T>(I, (unsigned)(I.S * I.nx), st, spec, I.xi[I.cur].as<T>(), dst, pa, ua, I.partials.as<double>());
}

template <typename T>
pfdd_status get_state_impl(pfdd_gpu *h, Instance &I, double *re, double *im, double *inter) {
  const size_t n = (size_t)I.S * I.N;
  if (h->staging.bytes < 2 * n * sizeof(double)) {
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->staging.release();
    CUDA_TRY(h, h->staging.alloc(2 * n * sizeof(double)));
  }
  DevBuf &tmp = h->staging;
  const T *dre = I.xi[I.cur].as<T>();
  const T *dim = I.F > I.S ? dre + n : nullptr;
  const bool synth = I.imag == IMAG_NYQ && (inter || im);
  if (synth) {
    // the other ping-pong buffer is free between steps
    ARM_FLAGS(h, I);
    T *scratch = I.xi[I.cur ^ 1].as<T>();
    synth_imag<T>(I, h->stream, scratch);
    dim = scratch;
  }
  if (inter) {
    k_to_interleaved<T><<<1184, 256, 0, h->stream>>>(dre, dim, tmp.as<double>(), n);
    CUDA_TRY(h, cudaMemcpyAsync(inter, tmp.p, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  } else {
    if (re) {
      k_to_planar<T><<<1184, 256, 0, h->stream>>>(dre, tmp.as<double>(), n);
      CUDA_TRY(h, cudaMemcpyAsync(re, tmp.p, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    if (im) {
      if (dim) {
        k_to_planar<T><<<1184, 256, 0, h->stream>>>(dim, tmp.as<double>() + n, n);
        CUDA_TRY(h, cudaMemcpyAsync(im, tmp.as<double>() + n, n * sizeof(double), cudaMemcpyDeviceToHost,
                                    h->stream));
      } else {
        memset(im, 0, n * sizeof(double));
      }
    }
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  CUDA_TRY(h, cudaGetLastError());
  if (synth) {
    int fl[4];
    CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
    if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
  }
  return PFDD_OK;
}

// whole-plane shared memory above which planes are split (two such CTAs
// cannot share an SM's 228 KB)
constexpr size_t kSplitAbove = 113 * 1024;

bool valid_size(int n) {
  if (n < 2 || n > 1024 || (n & 1)) return false;
  FftPlan p;
  return make_plan(n, p) && make_plan(n / 2, p);
}

}  // namespace

// Measured choice of the x-pencil tile width per group: every width the
// group's grid divides into and shared memory holds is timed on the device
// (CUDA events, `reps` launches after one warm-up) and the fastest kept.  The
// trial launches overwrite the spectrum buffer, which holds no state between
// calls (every advance opens with a forward pass), and the Nyquist carriers
// and stop flags, which are saved and restored.  Captured graphs are dropped.
template <typename T>
pfdd_status autotune_impl(pfdd_gpu *h, int reps, int *chosen) {
  constexpr int NC = Threads<T>::pencil;
  cudaStream_t st = h->stream;
  CUDA_TRY(h, cudaStreamSynchronize(st));
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  cudaEvent_t e0, e1;
  CUDA_TRY(h, cudaEventCreate(&e0));
  CUDA_TRY(h, cudaEventCreate(&e1));
  struct Ev {
    cudaEvent_t a, b;
    ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } guard{e0, e1};
  auto apply = [&](const Group &G, int cc) -> pfdd_status {
    for (int m : G.members) {
      Instance &I = *h->inst[m];
      const size_t ncols = (size_t)I.ny * I.nzp;
      I.ccols = cc;
      I.fstride = pencil_fstride<T>(I, cc);
      I.ntiles = (int)(ncols / cc);
      I.smem_pencil = pencil_smem<T>(I, cc);
      if (I.imag == IMAG_NYQ && I.ppart.bytes < 2 * (size_t)I.ntiles * sizeof(double)) {
        I.ppart.release();
        CUDA_TRY(h, I.ppart.alloc(2 * (size_t)I.ntiles * sizeof(double)));
      }
    }
    cudaError_t e = cudaSuccess;
    with_pencil_sc(h->inst[G.members[0]]->S, [&](auto SCc) {
      constexpr int SC = decltype(SCc)::value;
      const size_t b = h->inst[G.members[0]]->smem_pencil;
      if (e == cudaSuccess) e = raise_smem_limit(k_xpencil<T, NC, SC>, b);
      if (e == cudaSuccess) e = raise_smem_limit(k_xpencil_tab<T, NC, SC>, b);
    });
    CUDA_TRY(h, e);
    return refresh_tables(h);
  };
  for (size_t gi = 0; gi < h->groups.size(); ++gi) {
    const Group &G = h->groups[gi];
    Instance &L = *h->inst[G.members[0]];
    // live state the trial launches touch
    std::vector<std::vector<unsigned char>> aux(G.members.size());
    std::vector<int> stop(G.members.size());
    for (size_t k = 0; k < G.members.size(); ++k) {
      Instance &I = *h->inst[G.members[k]];
      if (I.aux.bytes) {
        aux[k].resize(I.aux.bytes);
        CUDA_TRY(h, cudaMemcpy(aux[k].data(), I.aux.p, I.aux.bytes, cudaMemcpyDeviceToHost));
      }
      CUDA_TRY(h, cudaMemcpy(&stop[k], I.flags(), sizeof(int), cudaMemcpyDeviceToHost));
      CUDA_TRY(h, cudaMemset(I.flags(), 0, sizeof(int)));
    }
    const size_t ncols = (size_t)L.ny * L.nzp;
    int best = L.ccols;
    float best_ms = 0.0f;
    for (int cc = 32; cc >= pencil_cmin<T>(); cc >>= 1) {
      if (ncols % cc || pencil_smem<T>(L, cc) > 227 * 1024) continue;
      pfdd_status ps = apply(G, cc);
      if (ps != PFDD_OK) return ps;
      launch_group_pencil<T>(L, G, st);
      CUDA_TRY(h, cudaEventRecord(e0, st));
      for (int r = 0; r < reps; ++r) launch_group_pencil<T>(L, G, st);
      CUDA_TRY(h, cudaEventRecord(e1, st));
      CUDA_TRY(h, cudaEventSynchronize(e1));
      CUDA_TRY(h, cudaGetLastError());
      float ms = 0.0f;
      CUDA_TRY(h, cudaEventElapsedTime(&ms, e0, e1));
      if (best_ms == 0.0f || ms < best_ms) {
        best_ms = ms;
        best = cc;
      }
    }
    pfdd_status ps = apply(G, best);
    if (ps != PFDD_OK) return ps;
    for (size_t k = 0; k < G.members.size(); ++k) {
      Instance &I = *h->inst[G.members[k]];
      if (I.aux.bytes) CUDA_TRY(h, cudaMemcpy(I.aux.p, aux[k].data(), I.aux.bytes, cudaMemcpyHostToDevice));
      CUDA_TRY(h, cudaMemcpy(I.flags(), &stop[k], sizeof(int), cudaMemcpyHostToDevice));
      if (chosen) chosen[G.members[k]] = best;
    }
  }
  return PFDD_OK;
}

template <typename T>
pfdd_status snapshot_begin_impl(pfdd_gpu *h, Instance &I, double *re, double *im) {
  const size_t n = (size_t)I.S * I.N;
  if (!h->copy_stream) CUDA_TRY(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  if (!I.snap.p) {
    CUDA_TRY(h, I.snap.alloc(2 * n * sizeof(double)));
    h->device_bytes += I.snap.bytes;
    CUDA_TRY(h, cudaEventCreateWithFlags(&I.snap_ready, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&I.snap_done, cudaEventDisableTiming));
  }
  // the previous snapshot's copies read I.snap: the conversion waits for them
  if (I.snap_pending) CUDA_TRY(h, cudaStreamWaitEvent(h->stream, I.snap_done, 0));
  const T *dre = I.xi[I.cur].as<T>();
  const T *dim = I.F > I.S ? dre + n : nullptr;
  if (I.imag == IMAG_NYQ && im) {
    ARM_FLAGS(h, I);
    T *scratch = I.xi[I.cur ^ 1].as<T>();   // free between steps
    synth_imag<T>(I, h->stream, scratch);
    dim = scratch;
  }
  double *d = I.snap.as<double>();
  k_to_planar<T><<<1184, 256, 0, h->stream>>>(dre, d, n);
  if (im) {
    if (dim) k_to_planar<T><<<1184, 256, 0, h->stream>>>(dim, d + n, n);
    else CUDA_TRY(h, cudaMemsetAsync(d + n, 0, n * sizeof(double), h->stream));
  }
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaEventRecord(I.snap_ready, h->stream));
  CUDA_TRY(h, cudaStreamWaitEvent(h->copy_stream, I.snap_ready, 0));
  if (re) CUDA_TRY(h, cudaMemcpyAsync(re, d, n * sizeof(double), cudaMemcpyDeviceToHost, h->copy_stream));
  if (im) CUDA_TRY(h, cudaMemcpyAsync(im, d + n, n * sizeof(double), cudaMemcpyDeviceToHost, h->copy_stream));
  CUDA_TRY(h, cudaEventRecord(I.snap_done, h->copy_stream));
  I.snap_pending = true;
  return PFDD_OK;
}

// ------------------------------------------------------------ checkpoints
// Index in the frequency-ordered carrier of a checkpoint file (kz = nz/2
// plane [S][kx][ky], ky = ny/2 plane [S][kx][kz], kx = nx/2 plane [S][ky][kz])
// of every complex value of the device's carrier, which is stored in
// transform-slot coordinates (the digit-reversed slots of this instance's
// plans; a split plane's rank r holds ky = r + 2k).
std::vector<size_t> carrier_file_order(const Instance &I) {
  const int nx = I.nx, ny = I.ny, M = I.M, S = I.S;
  std::vector<int> fx(nx), fy(ny), fz(M);
  const std::vector<int> px = positions(I.px), py = positions(I.py), pz = positions(I.pz);
  for (int k = 0; k < nx; ++k) fx[px[k]] = k;
  if (I.split) {
    const int nyh = ny / 2;
    for (int r = 0; r < 2; ++r)
      for (int k = 0; k < nyh; ++k) fy[r * nyh + py[k]] = r + 2 * k;
  } else {
    for (int k = 0; k < ny; ++k) fy[py[k]] = k;
  }
  for (int k = 0; k < M; ++k) fz[pz[k]] = k;
  std::vector<size_t> out;
  out.reserve((size_t)S * ((size_t)nx * ny + (size_t)nx * M + (size_t)ny * M));
  const size_t oZ = 0, oY = (size_t)S * nx * ny, oX = oY + (size_t)S * nx * M;
  for (int f = 0; f < S; ++f)
    for (int sx = 0; sx < nx; ++sx)
      for (int sy = 0; sy < ny; ++sy) out.push_back(oZ + ((size_t)f * nx + fx[sx]) * ny + fy[sy]);
  for (int f = 0; f < S; ++f)
    for (int sx = 0; sx < nx; ++sx)
      for (int sz = 0; sz < M; ++sz) out.push_back(oY + ((size_t)f * nx + fx[sx]) * M + fz[sz]);
  for (int f = 0; f < S; ++f)
    for (int sy = 0; sy < ny; ++sy)
      for (int sz = 0; sz < M; ++sz) out.push_back(oX + ((size_t)f * ny + fy[sy]) * M + fz[sz]);
  return out;
}

template <typename T>
pfdd_status checkpoint_save_impl(pfdd_gpu *h, Instance &I, const char *path) {
  pfdd_checkpoint_info in;
  memset(&in, 0, sizeof in);
  in.nx = I.nx; in.ny = I.ny; in.nz = I.nz; in.n_slip = I.S; in.fields = I.F;
  in.precision = sizeof(T) == 8 ? PFDD_FP64 : PFDD_FP32;
  in.imag_mode = I.imag == IMAG_FULL ? PFDD_IMAG_FULL : PFDD_IMAG_NYQUIST;
  in.advanced = I.advanced ? 1 : 0;
  in.field_bytes = (size_t)I.F * I.N * sizeof(T);
  in.carrier_bytes = I.imag == IMAG_NYQ ? I.aux.bytes : 0;
  in.steps = I.steps_total;
  std::vector<unsigned char> f(in.field_bytes), c(in.carrier_bytes);
  double sig[18];
  CUDA_TRY(h, cudaMemcpyAsync(f.data(), I.xi[I.cur].p, in.field_bytes, cudaMemcpyDeviceToHost, h->stream));
  if (in.carrier_bytes)
    CUDA_TRY(h, cudaMemcpyAsync(c.data(), I.aux.p, in.carrier_bytes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(sig, I.sigma(), sizeof sig, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int i = 0; i < 9; ++i) {
    in.sigma[i / 3][i % 3] = sig[i];
    in.dsigma[i / 3][i % 3] = sig[9 + i];
  }
  if (!c.empty()) {   // slot order -> the file's frequency order
    const std::vector<size_t> ord = carrier_file_order(I);
    if (ord.size() * sizeof(cx<T>) != c.size()) return fail(h, PFDD_EINVAL, "carrier size mismatch");
    std::vector<unsigned char> cf(c.size());
    for (size_t i = 0; i < ord.size(); ++i) memcpy(&cf[ord[i] * sizeof(cx<T>)], &c[i * sizeof(cx<T>)], sizeof(cx<T>));
    c.swap(cf);
  }
  const pfdd_status st = pfdd_checkpoint_write(path, &in, f.data(), c.empty() ? nullptr : c.data());
  if (st != PFDD_OK) return fail(h, st, "cannot write checkpoint %s", path);
  return PFDD_OK;
}

template <typename T>
pfdd_status checkpoint_load_impl(pfdd_gpu *h, Instance &I, const char *path) {
  pfdd_checkpoint_info in;
  if (pfdd_checkpoint_read(path, &in, nullptr, 0, nullptr, 0) != PFDD_OK)
    return fail(h, PFDD_EINVAL, "%s is not a readable checkpoint", path);
  const int want_imag = I.imag == IMAG_FULL ? PFDD_IMAG_FULL : PFDD_IMAG_NYQUIST;
  const size_t fb = (size_t)I.F * I.N * sizeof(T), cb = I.imag == IMAG_NYQ ? I.aux.bytes : 0;
  if (in.nx != I.nx || in.ny != I.ny || in.nz != I.nz || in.n_slip != I.S || in.fields != I.F ||
      in.precision != (sizeof(T) == 8 ? PFDD_FP64 : PFDD_FP32) || in.imag_mode != want_imag ||
      in.field_bytes != fb || in.carrier_bytes != cb)
    return fail(h, PFDD_EINVAL, "checkpoint %s was written for another grid, precision or carrier", path);
  std::vector<unsigned char> f(fb), c(cb);
  if (pfdd_checkpoint_read(path, &in, f.data(), fb, c.empty() ? nullptr : c.data(), cb) != PFDD_OK)
    return fail(h, PFDD_EINVAL, "checkpoint %s is truncated or corrupted (checksum)", path);
  double sig[18];
  for (int i = 0; i < 9; ++i) {
    sig[i] = in.sigma[i / 3][i % 3];
    sig[9 + i] = in.dsigma[i / 3][i % 3];
  }
  if (cb) {   // the file's frequency order -> this instance's slot order
    const std::vector<size_t> ord = carrier_file_order(I);
    if (ord.size() * sizeof(cx<T>) != cb) return fail(h, PFDD_EINVAL, "carrier size mismatch");
    std::vector<unsigned char> cs(cb);
    for (size_t i = 0; i < ord.size(); ++i) memcpy(&cs[i * sizeof(cx<T>)], &c[ord[i] * sizeof(cx<T>)], sizeof(cx<T>));
    c.swap(cs);
  }
  CUDA_TRY(h, cudaMemcpyAsync(I.xi[I.cur].p, f.data(), fb, cudaMemcpyHostToDevice, h->stream));
  if (cb) CUDA_TRY(h, cudaMemcpyAsync(I.aux.p, c.data(), cb, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(I.sigma(), sig, sizeof sig, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  I.advanced = in.advanced != 0;
  I.steps_total = in.steps;
  I.tape_steps = 0;
  return PFDD_OK;
}

template <typename T>
pfdd_status cond_step_impl(pfdd_gpu *h, Instance &I, int n_iters, pfdd_cond_stats *stats) {
  using C = cx<T>;
  constexpr int NP = Threads<T>::plane, NH = Threads<T>::half;
  cudaStream_t st = h->stream;
  ARM_FLAGS(h, I);
  const size_t N = I.N, ncols = (size_t)I.ny * I.nzp;
  const int nb = 2 * h->nsm;
  if (I.cond_part.bytes < (size_t)n_iters * nb * 3 * sizeof(double)) {
    CUDA_TRY(h, cudaStreamSynchronize(st));
    I.cond_part.release();
    CUDA_TRY(h, I.cond_part.alloc((size_t)n_iters * nb * 3 * sizeof(double)));
  }
  // pencil tile: the widest that holds four fields in shared memory
  int cc = I.ccols;
  auto bytes = [&](int c) { return ((size_t)4 * I.nx * c + I.nx) * sizeof(C); };
  while (cc > 1 && bytes(cc) > 227 * 1024) cc >>= 1;
  if (bytes(cc) > 227 * 1024 || ncols % cc)
    return fail(h, PFDD_EUNSUPPORTED, "conductivity pencil of %d x 4 fields does not fit shared memory", I.nx);
  CUDA_TRY(h, raise_smem_limit(k_cond_pencil<T, 256>, bytes(cc)));
  PlaneArgs pa;
  fill_plane_args<T>(I, pa);
  PencilArgs pe{};
  pe.px = I.px;
  pe.nx = I.nx; pe.ny = I.ny; pe.nz = I.nz; pe.nzh = I.nzh; pe.nzp = I.nzp; pe.M = I.M;
  pe.S = 1; pe.F = 2; pe.imag = IMAG_FULL;
  pe.ncols = (int)ncols;
  pe.ccols = cc;
  pe.tw_x = I.tw_x.p;
  pe.kx_of = I.kx_of; pe.ky_of = I.ky_of; pe.kz_of = I.kz_of;
  pe.mode = PASS_STEP;
  pe.fstride = I.nx * cc;
  pe.sx_n = I.sx_n; pe.sy_n = I.sy_n;
  pe.g = I.green;
  set_pencil_divisors<T>(pe);
  pe.fd_6cc = FastDiv(4 * cc);
  UpdateArgs ua;
  memset(&ua, 0, sizeof ua);
  ua.nx = I.nx; ua.ny = I.ny; ua.nz = I.nz; ua.nzh = I.nzh; ua.nzp = I.nzp; ua.S = I.S; ua.F = 4;
  ua.invN = 1.0;   // backwardcond's transforms are unnormalised
  ua.core = I.core;
  ua.err = I.flags() + 3;
  ua.mode = PASS_SYNTH;
  CondArgs ca;
  ca.El = I.cond_El;
  ca.eps0 = I.cond_eps0;
  ca.dt = I.cond_dt;
  ca.ny = I.ny;
  ca.nz = I.nz;
  const unsigned planes2 = (unsigned)(2 * I.nx), planes4 = (unsigned)(4 * I.nx);
  T *cxi = I.cond_xi.as<T>();
  for (int it = 0; it < n_iters; ++it) {
    pa.F = 2;
    if (I.split)
      launch_pair(k_fwd_planes<T, NH, true>, dim3(2 * planes2), NH, I.smem_plane, st, (const T *)cxi,
                  I.cond_in.as<C>(), pa, (const int *)nullptr, I.flags() + 3);
    else
      k_fwd_planes<T, NP, false><<<planes2, NP, I.smem_plane, st>>>(cxi, I.cond_in.as<C>(), pa, nullptr,
                                                                     I.flags() + 3);
    k_cond_pencil<T, 256><<<(unsigned)(ncols / cc), 256, bytes(cc), st>>>(I.cond_in.as<C>(), I.cond_out.as<C>(), pe);
    pa.F = 4;
    if (I.split)
      launch_pair(k_inv_update<T, NH, true>, dim3(2 * planes4), NH, I.smem_update, st,
                  (const C *)I.cond_out.as<C>(), (const T *)cxi, I.cond_real.as<T>(), pa, ua, I.partials.as<double>());
    else
      k_inv_update<T, NP, false><<<planes4, NP, I.smem_update, st>>>(I.cond_out.as<C>(), cxi, I.cond_real.as<T>(),
                                                                     pa, ua, I.partials.as<double>());
    k_cond_update<T><<<nb, 256, 0, st>>>(cxi, I.cond_real.as<T>(), I.cond_tab.as<double>(), ca, N,
                                          I.cond_part.as<double>() + (size_t)it * nb * 3);
    CUDA_TRY(h, cudaGetLastError());
  }
  std::vector<double> hp((size_t)n_iters * nb * 3);
  CUDA_TRY(h, cudaMemcpyAsync(hp.data(), I.cond_part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  int fl[4];
  CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
  if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
  if (stats) {
    for (int it = 0; it < n_iters; ++it) {
      double tot[3];
      for (int q = 0; q < 3; ++q) {
        double t = 0.0, c = 0.0;
        for (int b = 0; b < nb; ++b) {   // Neumaier-compensated
          const double v = hp[((size_t)it * nb + b) * 3 + q], u = t + v;
          c += (std::fabs(t) >= std::fabs(v)) ? (t - u) + v : (v - u) + t;
          t = u;
        }
        tot[q] = t + c;
      }
      stats[it].condxinorm = std::sqrt(tot[0]);
      stats[it].condxiave = tot[1];
      stats[it].conductivity = tot[2] / (1.0 * I.cond_El);
    }
  }
  return PFDD_OK;
}

extern "C" {

const char *pfdd_gpu_version(void) { return "pfdd_b200 0.1 (sm_100a)"; }

pfdd_status pfdd_gpu_create(const pfdd_instance_desc *descs, int n_instances, const pfdd_options *opt,
                            pfdd_gpu **out) {
  if (!out) return fail(nullptr, PFDD_EINVAL, "out is NULL");
  *out = nullptr;
  if (!descs || n_instances < 1) return fail(nullptr, PFDD_EINVAL, "need at least one instance");
  pfdd_options o{};
  o.precision = PFDD_FP64;
  o.imag_mode = PFDD_IMAG_AUTO;
  o.use_graphs = 1;
  o.check_finite = 1;
  if (opt) o = *opt;
  if (o.precision != PFDD_FP64 && o.precision != PFDD_FP32)
    return fail(nullptr, PFDD_EINVAL, "precision must be PFDD_FP64 or PFDD_FP32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, PFDD_ENODEVICE, "no CUDA device");
  if (o.device < 0 || o.device >= ndev) return fail(nullptr, PFDD_EINVAL, "device %d out of range", o.device);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess || prop.major < 10)
    return fail(nullptr, PFDD_ENODEVICE, "device %d is not sm_100 class", o.device);
  for (int i = 0; i < n_instances; ++i) {
    const pfdd_instance_desc &d = descs[i];
    if (d.n_slip < 1 || d.n_slip > PFDD_MAX_SLIP)
      return fail(nullptr, PFDD_EINVAL, "instance %d: n_slip %d outside 1..%d", i, d.n_slip, PFDD_MAX_SLIP);
    if (!valid_size(d.nx) || !valid_size(d.ny) || !valid_size(d.nz) || d.nz % 4)
      return fail(nullptr, PFDD_EUNSUPPORTED,
                  "instance %d: grid %dx%dx%d: each extent must be even and 2^a 3^b, <= 1024, nz a multiple of 4",
                  i, d.nx, d.ny, d.nz);
    if (!(d.dslip > 0) || !(d.b > 0) || !(d.C44 > 0))
      return fail(nullptr, PFDD_EINVAL, "instance %d: dslip, b and C44 must be positive", i);
  }
  std::unique_ptr<pfdd_gpu> h(new pfdd_gpu);
  h->opt = o;
  h->precision = o.precision;
  h->device = o.device;
  h->nsm = prop.multiProcessorCount;
  if (cudaSetDevice(o.device) != cudaSuccess) return fail(nullptr, PFDD_ECUDA, "cudaSetDevice failed");
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(nullptr, PFDD_ECUDA, "stream creation failed");
  h->stream = h->own_stream;
  // Mixed-size batches: instances whose descriptors differ only in the grid
  // size, when the batch holds two sizes or more, run their groups in one
  // launch per pass (whole planes; PFDD_MERGE=0 in the environment keeps one
  // launch per group).
  auto same_but_size = [&](const pfdd_instance_desc &x, const pfdd_instance_desc &y) {
    const int S = x.n_slip;
    return S == y.n_slip && x.core_flag == y.core_flag && x.C44 == y.C44 && x.C12 == y.C12 && x.C11 == y.C11 &&
           x.dslip == y.dslip && x.b == y.b && x.cd_dt == y.cd_dt && x.isf == y.isf && x.usf == y.usf &&
           x.An == y.An && !memcmp(x.four, y.four, sizeof x.four) && !memcmp(x.prim, y.prim, sizeof x.prim) &&
           !memcmp(x.xn, y.xn, sizeof(double) * 3 * S) && !memcmp(x.xb, y.xb, sizeof(double) * 3 * S) &&
           !memcmp(x.c, y.c, sizeof x.c) && !memcmp(x.aa, y.aa, sizeof x.aa) && !memcmp(x.bb, y.bb, sizeof x.bb) &&
           (x.non_schmid != 0) == (y.non_schmid != 0) && x.angle_to_110 == y.angle_to_110 && x.w1 == y.w1 &&
           x.w2 == y.w2 && x.w3 == y.w3 && !memcmp(x.usfe_fit, y.usfe_fit, sizeof x.usfe_fit) &&
           (x.xo == nullptr) == (y.xo == nullptr) && (x.site_gsfe == nullptr) == (y.site_gsfe == nullptr);
  };
  std::vector<char> batch_mixed(n_instances, 0);
  {
    const char *env = getenv("PFDD_MERGE");
    if (!(env && !strcmp(env, "0")))
      for (int i = 0; i < n_instances; ++i)
        for (int j = 0; j < n_instances && !batch_mixed[i]; ++j)
          if (same_but_size(descs[i], descs[j]) &&
              (descs[i].nx != descs[j].nx || descs[i].ny != descs[j].ny || descs[i].nz != descs[j].nz))
            batch_mixed[i] = 1;
  }
  size_t max_plane = 0, max_upd = 0, max_pen = 0;
  for (int i = 0; i < n_instances; ++i) {
    std::unique_ptr<Instance> I(new Instance);
    I->d = descs[i];
    I->d.site_gsfe = nullptr;
    I->d.xo = nullptr;
    I->S = descs[i].n_slip;
    int imag = o.imag_mode;
    if (imag == PFDD_IMAG_AUTO) imag = descs[i].xo ? PFDD_IMAG_FULL : PFDD_IMAG_NYQUIST;
    if (imag == PFDD_IMAG_NYQUIST && descs[i].xo)
      return fail(nullptr, PFDD_EINVAL, "instance %d: PFDD_IMAG_NYQUIST is exact only without an obstacle mask", i);
    if (imag != PFDD_IMAG_FULL && imag != PFDD_IMAG_NYQUIST)
      return fail(nullptr, PFDD_EINVAL, "instance %d: unknown imag_mode %d", i, imag);
    I->imag = (imag == PFDD_IMAG_FULL) ? IMAG_FULL : IMAG_NYQ;
    I->F = I->imag == IMAG_FULL ? 2 * I->S : I->S;
    I->nx = descs[i].nx; I->ny = descs[i].ny; I->nz = descs[i].nz;
    I->M = I->nz / 2;
    I->nzh = I->M + 1;
    // spectrum rows padded to whole 16-byte units so a plane moves in one bulk copy
    I->nzp = (o.precision == PFDD_FP32) ? ((I->nzh + 1) & ~1) : I->nzh;
    // shared-memory row stride: FP32 rows start 4 words apart in the 32 banks
    // (2*nzs = 4 mod 32), which the register-resident z passes' thread order
    // turns into conflict-free block loads; FP64: nzs = 4 mod 8 16-byte units
    I->nzs = I->nzp;
    if (o.precision == PFDD_FP32)
      while ((2 * I->nzs) % 32 != 4) I->nzs += 2;
    else
      while (I->nzs % 8 != 4) ++I->nzs;
    // store spectrum rows with the same stride, so a plane moves in one bulk copy
    I->nzp = I->nzs;
    I->N = (size_t)I->nx * I->ny * I->nz;
    // Split the P1/P3 planes over 2-CTA clusters when a whole plane leaves
    // room for one CTA per SM only (or does not fit); PFDD_PLANE_SPLIT=0|1
    // in the environment forces the choice.
    const size_t whole = (o.precision == PFDD_FP32) ? PlaneSmem<cx<float>>::bytes(I->ny, I->ny, I->nzs, I->M)
                                                    : PlaneSmem<cx<double>>::bytes(I->ny, I->ny, I->nzs, I->M);
    // (small grids split too, so the plane passes fill the SMs twice over)
    I->split = whole > kSplitAbove || I->F * I->nx < 2 * h->nsm;
    if (batch_mixed[i] && whole <= kSplitAbove) {   // a batch fills the SMs by instance count
      I->split = false;
      I->merged = true;
    }
    if (const char *env = getenv("PFDD_PLANE_SPLIT")) {
      if (!strcmp(env, "0")) I->split = false;
      else if (!strcmp(env, "1")) I->split = true;
    }
    // PFDD_ZFUSED=0: the update and adjoint passes keep the generic staged z
    // passes (same results to round-off; the tests compare the two)
    if (const char *env = getenv("PFDD_ZFUSED")) I->zfused = strcmp(env, "0") ? 1 : 0;
    const int maxr = (o.precision == PFDD_FP32)
                         ? std::min(MaxRadix<Threads<float>::plane>::value, MaxRadix<Threads<float>::half>::value)
                         : std::min(MaxRadix<Threads<double>::plane>::value, MaxRadix<Threads<double>::half>::value);
    make_plan(I->nx, I->px, maxr);
    make_plan(I->split ? I->ny / 2 : I->ny, I->py, maxr);
    make_zplan(I->M, I->pz, maxr);
    pfdd_instance_desc d = descs[i];
    I->d.xo = d.xo;               // used during set-up only
    I->d.site_gsfe = d.site_gsfe;
    pfdd_status st = (o.precision == PFDD_FP64) ? setup_instance<double>(h.get(), *I) : setup_instance<float>(h.get(), *I);
    I->d.xo = nullptr;
    I->d.site_gsfe = nullptr;
    if (st != PFDD_OK) {
      g_create_error = h->err;
      return st;
    }
    max_plane = std::max(max_plane, I->smem_plane);
    max_upd = std::max(max_upd, I->smem_update);
    max_pen = std::max(max_pen, I->smem_pencil);
    h->inst.push_back(std::move(I));
  }
  pfdd_status st = (o.precision == PFDD_FP64) ? set_smem_attrs<double>(h.get(), max_plane, max_upd, max_pen)
                                              : set_smem_attrs<float>(h.get(), max_plane, max_upd, max_pen);
  if (st != PFDD_OK) { g_create_error = h->err; return st; }
  build_groups(h.get());
  if ((st = ensure_stats(h.get(), 1)) != PFDD_OK || (st = refresh_tables(h.get())) != PFDD_OK) {
    g_create_error = h->err;
    return st;
  }
  *out = h.release();
  return PFDD_OK;
}

pfdd_status pfdd_gpu_set_state(pfdd_gpu *h, int inst, const double *xi_re, const double *xi_im) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  if (!xi_re) return fail(h, PFDD_EINVAL, "xi_re is NULL");
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? set_state_impl<double>(h, *h->inst[inst], xi_re, xi_im, false)
                                   : set_state_impl<float>(h, *h->inst[inst], xi_re, xi_im, false);
}

pfdd_status pfdd_gpu_set_state_interleaved(pfdd_gpu *h, int inst, const double *xi) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  if (!xi) return fail(h, PFDD_EINVAL, "xi is NULL");
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? set_state_impl<double>(h, *h->inst[inst], xi, nullptr, true)
                                   : set_state_impl<float>(h, *h->inst[inst], xi, nullptr, true);
}

pfdd_status pfdd_gpu_get_state(pfdd_gpu *h, int inst, double *xi_re, double *xi_im) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? get_state_impl<double>(h, *h->inst[inst], xi_re, xi_im, nullptr)
                                   : get_state_impl<float>(h, *h->inst[inst], xi_re, xi_im, nullptr);
}

pfdd_status pfdd_gpu_get_state_interleaved(pfdd_gpu *h, int inst, double *xi) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  if (!xi) return fail(h, PFDD_EINVAL, "xi is NULL");
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? get_state_impl<double>(h, *h->inst[inst], nullptr, nullptr, xi)
                                   : get_state_impl<float>(h, *h->inst[inst], nullptr, nullptr, xi);
}

pfdd_status pfdd_gpu_advance(pfdd_gpu *h, int n_steps, int stress_states, double tol, pfdd_step_stats *stats) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (n_steps < 0 || stress_states < 0) return fail(h, PFDD_EINVAL, "negative step count");
  if (n_steps == 0 || stress_states == 0) return PFDD_OK;
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? advance_impl<double>(h, n_steps, stress_states, tol, stats)
                                   : advance_impl<float>(h, n_steps, stress_states, tol, stats);
}

pfdd_status pfdd_gpu_step_history(pfdd_gpu *h, int inst, double *xinorm, double *xiave, int cap, int *count) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  Instance &I = *h->inst[inst];
  const int n = std::min(cap, I.hist_count);
  for (int i = 0; i < n; ++i) {
    if (xinorm) xinorm[i] = I.hist[2 * i];
    if (xiave) xiave[i] = I.hist[2 * i + 1];
  }
  if (count) *count = I.hist_count;
  return PFDD_OK;
}

pfdd_status pfdd_gpu_checkpoint_save(pfdd_gpu *h, int inst, const char *path) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size() || !path) return fail(h, PFDD_EINVAL, "bad arguments");
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? checkpoint_save_impl<double>(h, *h->inst[inst], path)
                                   : checkpoint_save_impl<float>(h, *h->inst[inst], path);
}

pfdd_status pfdd_gpu_checkpoint_load(pfdd_gpu *h, int inst, const char *path) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size() || !path) return fail(h, PFDD_EINVAL, "bad arguments");
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? checkpoint_load_impl<double>(h, *h->inst[inst], path)
                                   : checkpoint_load_impl<float>(h, *h->inst[inst], path);
}

pfdd_status pfdd_gpu_set_stress(pfdd_gpu *h, int inst, const double sigma[3][3]) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size() || !sigma) return fail(h, PFDD_EINVAL, "bad arguments");
  Instance &I = *h->inst[inst];
  cudaSetDevice(h->device);
  double s[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      if (!std::isfinite(sigma[i][j])) return fail(h, PFDD_EINVAL, "non-finite sigma");
      s[3 * i + j] = sigma[i][j];
    }
  CUDA_TRY(h, cudaMemcpyAsync(I.sigma(), s, sizeof s, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  I.advanced = false;   // the device sigma is the current stress state again
  return PFDD_OK;
}

pfdd_status pfdd_gpu_tau(pfdd_gpu *h, int inst, double *tau) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size() || !tau) return fail(h, PFDD_EINVAL, "bad arguments");
  Instance &I = *h->inst[inst];
  cudaSetDevice(h->device);
  k_stress_state<<<1, 32, 0, h->stream>>>(I.sigma(), I.tau(), I.an(), I.stress, 0, nullptr);
  CUDA_TRY(h, cudaMemcpyAsync(tau, I.tau(), I.S * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return PFDD_OK;
}

pfdd_status pfdd_gpu_energy(pfdd_gpu *h, int inst, double *e_elastic, double *e_core, double *e_applied) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  Instance &I = *h->inst[inst];
  const int f = I.d.core_flag;
  if (f == PFDD_CORE_PYRII)
    return fail(h, PFDD_EUNSUPPORTED, "no energy density for core model %d", f);
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? energy_impl<double>(h, I, e_elastic, e_core, e_applied)
                                   : energy_impl<float>(h, I, e_elastic, e_core, e_applied);
}

pfdd_status pfdd_gpu_strain_stress(pfdd_gpu *h, int inst, double *eps, double *sigma, double *ave_eps,
                                   double *ave_sigma) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? strain_stress_impl<double>(h, *h->inst[inst], eps, sigma, ave_eps, ave_sigma)
                                   : strain_stress_impl<float>(h, *h->inst[inst], eps, sigma, ave_eps, ave_sigma);
}

pfdd_status pfdd_gpu_core_profile(pfdd_gpu *h, int inst, int n_planes, double *delta, double *ddelta) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  Instance &I = *h->inst[inst];
  if (!delta || n_planes < 1 || (I.S <= 2 ? n_planes > I.S : 3 * n_planes > I.S))
    return fail(h, PFDD_EINVAL, "need delta and 1 <= n_planes <= %d", I.S <= 2 ? I.S : I.S / 3);
  cudaSetDevice(h->device);
  cudaStream_t st = h->stream;
  const size_t n = (size_t)n_planes * I.N;
  DevBuf out;
  CUDA_TRY(h, out.alloc(n * sizeof(double)));
  ProfileArgs pa;
  memset(&pa, 0, sizeof pa);
  for (int a = 0; a < 3 && a < I.S; ++a)
    for (int c = 0; c < 3; ++c) pa.xb[a][c] = I.d.xb[a][c];
  const int blocks = 4 * h->nsm;
  if (h->precision == PFDD_FP64)
    k_core_profile<double><<<blocks, 256, 0, st>>>(I.xi[I.cur].as<double>(), I.S, I.N, n_planes, pa, out.as<double>());
  else
    k_core_profile<float><<<blocks, 256, 0, st>>>(I.xi[I.cur].as<float>(), I.S, I.N, n_planes, pa, out.as<double>());
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaMemcpyAsync(delta, out.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(h, cudaStreamSynchronize(st));
  if (ddelta) {
    // the line j = ny/2, k = nz/2: forward difference with dx = nx/nx = 1 (fft_fftw_slab.cpp:1597-1620)
    const size_t line = (size_t)(I.ny / 2) * I.nz + I.nz / 2, sx = (size_t)I.ny * I.nz;
    for (int p = 0; p < n_planes; ++p)
      for (int i = 0; i < I.nx; ++i) {
        const double *d = delta + (size_t)p * I.N + line;
        const double here = d[(size_t)i * sx], next = (i + 1 < I.nx) ? d[(size_t)(i + 1) * sx] : here;
        ddelta[(size_t)p * I.nx + i] = (next - here) / 1.0;
      }
  }
  return PFDD_OK;
}

pfdd_status pfdd_cond_layers(const pfdd_cond_material *A, const pfdd_cond_material *B, int ny, double temperature,
                             double *sigma_eff, double *sigma_layer) {
  if (!A || !B || !sigma_eff || !sigma_layer || ny < 1 || A->Nlayers < 1)
    return fail(nullptr, PFDD_EINVAL, "need A, B, outputs, ny >= 1 and A->Nlayers >= 1");
  // backwardcond (fft_fftw_slab.cpp:2089-2156), in its order of operations
  const double Vf = B->dlayer / (A->dlayer + B->dlayer);
  const double prob = 1.0 - A->pinterface;
  const int per = ny / A->Nlayers;
  const int dB = (int)std::round(per * Vf), dA = (int)std::round(per * (1. - Vf));
  if (dA + dB < 1) return fail(nullptr, PFDD_EINVAL, "layer period of zero cells (ny / Nlayers too small)");
  const double dT = temperature - 300;
  for (int j = 0; j < ny; ++j) {
    const pfdd_cond_material &M = (j % (dA + dB) >= dA) ? *B : *A;
    const double lay = M.condsigma / (1. + M.alpha_resistivity * dT);
    const double ps = 2 * prob / M.dlayer;
    const double lam = M.mfpel / (1. + M.alpha_mfpel * dT);
    const double ag = (lam * M.Ngrains / M.dlayer) * M.Rgrain / (1 - M.Rgrain);
    const double rd = M.beta_disloc * M.rho_disloc;
    double cs;
    if (ps > 0.) {
      const double ri = ((1 / lay) * ((3. / 16.) * lam * ps));
      if (M.Ngrains > 1) {
        const double rg =
            (1 / lay) * (1. / (1. - 3. * ag / 2. + 3. * ag * ag - 3. * std::pow(ag, 3.) * std::log(1. + 1. / ag)) - 1.);
        cs = 1 / ((1 / lay) + (2 * ri + (M.Ngrains - 1) * rg) / (M.Ngrains + 1) + rd);
      } else {
        cs = 1 / ((1 / lay) + ri + rd);
      }
    } else {
      cs = lay;
    }
    sigma_eff[j] = cs;
    sigma_layer[j] = lay;
  }
  return PFDD_OK;
}

pfdd_status pfdd_gpu_cond_enable(pfdd_gpu *h, int inst, const pfdd_cond_desc *d) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  Instance &I = *h->inst[inst];
  if (!d || !d->sigma_eff || !d->sigma_layer) return fail(h, PFDD_EINVAL, "need the per-y conductivity tables");
  if (I.ny < 2) return fail(h, PFDD_EINVAL, "the conductivity gradient needs ny >= 2");
  cudaSetDevice(h->device);
  const size_t TB = h->precision == PFDD_FP64 ? sizeof(double) : sizeof(float);
  const size_t CB = 2 * TB, ncols = (size_t)I.ny * I.nzp;
  if (!I.cond_on) {
    CUDA_TRY(h, I.cond_xi.alloc(2 * I.N * TB));
    CUDA_TRY(h, I.cond_in.alloc(2 * (size_t)I.nx * ncols * CB));
    CUDA_TRY(h, I.cond_out.alloc(4 * (size_t)I.nx * ncols * CB));
    CUDA_TRY(h, I.cond_real.alloc(4 * I.N * TB));
    CUDA_TRY(h, I.cond_tab.alloc(2 * (size_t)I.ny * sizeof(double)));
    h->device_bytes += I.cond_xi.bytes + I.cond_in.bytes + I.cond_out.bytes + I.cond_real.bytes + I.cond_tab.bytes;
  }
  // d sigma_layer / dy as backwardcond takes it (one-sided at the ends, :2170-2183)
  std::vector<double> tab(2 * (size_t)I.ny);
  const double *L = d->sigma_layer;
  for (int j = 0; j < I.ny; ++j) {
    tab[j] = d->sigma_eff[j];
    tab[I.ny + j] = (j == 0) ? (L[j + 1] - L[j]) : (j == I.ny - 1) ? (L[j] - L[j - 1]) : (L[j + 1] - L[j - 1]) / 2.;
  }
  CUDA_TRY(h, cudaMemcpy(I.cond_tab.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemset(I.cond_xi.p, 0, I.cond_xi.bytes));
  I.cond_El = d->El_y;
  I.cond_eps0 = d->epsilonzero;
  I.cond_dt = d->timestep;
  I.cond_on = true;
  return PFDD_OK;
}

pfdd_status pfdd_gpu_cond_set_state(pfdd_gpu *h, int inst, const double *re, const double *im) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  Instance &I = *h->inst[inst];
  if (!I.cond_on) return fail(h, PFDD_ESTATE, "pfdd_gpu_cond_enable has not been called for instance %d", inst);
  if (!re) return fail(h, PFDD_EINVAL, "re is required");
  cudaSetDevice(h->device);
  if (h->precision == PFDD_FP64) {
    CUDA_TRY(h, cudaMemcpy(I.cond_xi.p, re, I.N * sizeof(double), cudaMemcpyHostToDevice));
    if (im) CUDA_TRY(h, cudaMemcpy(I.cond_xi.as<double>() + I.N, im, I.N * sizeof(double), cudaMemcpyHostToDevice));
    else CUDA_TRY(h, cudaMemset(I.cond_xi.as<double>() + I.N, 0, I.N * sizeof(double)));
  } else {
    std::vector<float> v(2 * I.N, 0.0f);
    for (size_t i = 0; i < I.N; ++i) {
      v[i] = (float)re[i];
      if (im) v[I.N + i] = (float)im[i];
    }
    CUDA_TRY(h, cudaMemcpy(I.cond_xi.p, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  return PFDD_OK;
}

pfdd_status pfdd_gpu_cond_get_state(pfdd_gpu *h, int inst, double *re, double *im) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  Instance &I = *h->inst[inst];
  if (!I.cond_on) return fail(h, PFDD_ESTATE, "pfdd_gpu_cond_enable has not been called for instance %d", inst);
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (h->precision == PFDD_FP64) {
    if (re) CUDA_TRY(h, cudaMemcpy(re, I.cond_xi.p, I.N * sizeof(double), cudaMemcpyDeviceToHost));
    if (im) CUDA_TRY(h, cudaMemcpy(im, I.cond_xi.as<double>() + I.N, I.N * sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    std::vector<float> v(2 * I.N);
    CUDA_TRY(h, cudaMemcpy(v.data(), I.cond_xi.p, v.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < I.N; ++i) {
      if (re) re[i] = v[i];
      if (im) im[i] = v[I.N + i];
    }
  }
  return PFDD_OK;
}

pfdd_status pfdd_gpu_autotune(pfdd_gpu *h, int reps, int *chosen) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (reps < 1) return fail(h, PFDD_EINVAL, "reps must be >= 1");
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? autotune_impl<double>(h, reps, chosen) : autotune_impl<float>(h, reps, chosen);
}

pfdd_status pfdd_gpu_snapshot_begin(pfdd_gpu *h, int inst, double *re, double *im) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  if (!re && !im) return fail(h, PFDD_EINVAL, "need re or im");
  cudaSetDevice(h->device);
  Instance &I = *h->inst[inst];
  return h->precision == PFDD_FP64 ? snapshot_begin_impl<double>(h, I, re, im)
                                   : snapshot_begin_impl<float>(h, I, re, im);
}

pfdd_status pfdd_gpu_snapshot_wait(pfdd_gpu *h, int inst) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  cudaSetDevice(h->device);
  Instance &I = *h->inst[inst];
  if (!I.snap_pending) return PFDD_OK;
  CUDA_TRY(h, cudaEventSynchronize(I.snap_done));
  I.snap_pending = false;
  CUDA_TRY(h, cudaGetLastError());
  int fl[4];
  CUDA_TRY(h, cudaMemcpy(fl, I.flags(), sizeof fl, cudaMemcpyDeviceToHost));
  if (fl[3]) return fail(h, PFDD_ETIMEOUT, "a bounded device wait ran out");
  return PFDD_OK;
}

pfdd_status pfdd_gpu_cond_step(pfdd_gpu *h, int inst, int n_iters, pfdd_cond_stats *stats) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  Instance &I = *h->inst[inst];
  if (!I.cond_on) return fail(h, PFDD_ESTATE, "pfdd_gpu_cond_enable has not been called for instance %d", inst);
  if (n_iters < 1) return fail(h, PFDD_EINVAL, "n_iters must be >= 1");
  cudaSetDevice(h->device);
  return h->precision == PFDD_FP64 ? cond_step_impl<double>(h, I, n_iters, stats)
                                   : cond_step_impl<float>(h, I, n_iters, stats);
}

static pfdd_status adjoint_check(pfdd_gpu *h, int inst) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (inst < 0 || inst >= (int)h->inst.size()) return fail(h, PFDD_EINVAL, "instance %d out of range", inst);
  const int f = h->inst[inst]->d.core_flag;
  if (f == PFDD_CORE_EXTENDED || f == PFDD_CORE_PYRII || f == PFDD_CORE_BCC_PERFECT)
    return fail(h, PFDD_EUNSUPPORTED, "no adjoint for core model %d", f);
  cudaSetDevice(h->device);
  return PFDD_OK;
}

pfdd_status pfdd_gpu_adjoint_forward(pfdd_gpu *h, int inst, int n_steps, int ckpt_every) {
  pfdd_status st = adjoint_check(h, inst);
  if (st != PFDD_OK) return st;
  if (n_steps < 1 || ckpt_every < 1) return fail(h, PFDD_EINVAL, "need n_steps, ckpt_every >= 1");
  Instance &I = *h->inst[inst];
  return h->precision == PFDD_FP64 ? adjoint_forward_impl<double>(h, I, n_steps, ckpt_every)
                                   : adjoint_forward_impl<float>(h, I, n_steps, ckpt_every);
}

pfdd_status pfdd_gpu_adjoint_backward(pfdd_gpu *h, int inst, const double *dL_dxiN, double *dL_dparams,
                                      double *dL_dsigma) {
  pfdd_status st = adjoint_check(h, inst);
  if (st != PFDD_OK) return st;
  if (!dL_dxiN) return fail(h, PFDD_EINVAL, "dL_dxiN is NULL");
  Instance &I = *h->inst[inst];
  return h->precision == PFDD_FP64 ? adjoint_backward_impl<double>(h, I, dL_dxiN, dL_dparams, dL_dsigma)
                                   : adjoint_backward_impl<float>(h, I, dL_dxiN, dL_dparams, dL_dsigma);
}

pfdd_status pfdd_gpu_adjoint(pfdd_gpu *h, int inst, int n_steps, int ckpt_every, const double *dL_dxiN,
                             double *dL_dparams, double *dL_dsigma) {
  if (h && !dL_dxiN) return fail(h, PFDD_EINVAL, "dL_dxiN is NULL");
  pfdd_status st = pfdd_gpu_adjoint_forward(h, inst, n_steps, ckpt_every);
  if (st != PFDD_OK) return st;
  return pfdd_gpu_adjoint_backward(h, inst, dL_dxiN, dL_dparams, dL_dsigma);
}

pfdd_status pfdd_gpu_set_stream(pfdd_gpu *h, void *stream) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  cudaSetDevice(h->device);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : h->own_stream;
  return PFDD_OK;
}

pfdd_status pfdd_gpu_profile(pfdd_gpu *h, int n_steps, double *kernel_ms, int *launches_per_step) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (n_steps < 1 || !kernel_ms) return fail(h, PFDD_EINVAL, "need n_steps >= 1 and kernel_ms");
  cudaSetDevice(h->device);
  if (launches_per_step) *launches_per_step = kLaunchesPerStep * n_units(h);
  return h->precision == PFDD_FP64 ? profile_impl<double>(h, n_steps, kernel_ms)
                                   : profile_impl<float>(h, n_steps, kernel_ms);
}

pfdd_status pfdd_gpu_info(pfdd_gpu *h, int *n_instances, size_t *device_bytes) {
  if (!h) return fail(nullptr, PFDD_EINVAL, "NULL handle");
  if (n_instances) *n_instances = (int)h->inst.size();
  if (device_bytes) *device_bytes = h->device_bytes;
  return PFDD_OK;
}

const char *pfdd_gpu_last_error(pfdd_gpu *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

void pfdd_gpu_destroy(pfdd_gpu *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  h->groups.clear();
  for (auto &ip : h->inst) {
    if (ip->snap_ready) cudaEventDestroy(ip->snap_ready);
    if (ip->snap_done) cudaEventDestroy(ip->snap_done);
  }
  h->inst.clear();
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->side_stream) {
    cudaStreamSynchronize(h->side_stream);
    cudaStreamDestroy(h->side_stream);
  }
  h->staging.release();
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  h->own_stream = nullptr;
  delete h;
}

}  // extern "C"
