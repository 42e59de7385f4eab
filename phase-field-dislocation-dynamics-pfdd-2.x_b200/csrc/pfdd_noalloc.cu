// pfdd_gl_step_noalloc: one FP64 Ginzburg-Landau iteration of one instance on
// caller-owned device buffers, without allocating any memory.
//
// Some callers cannot call cudaMalloc: host codes whose runtime hands out all
// device memory through its own pool and forbids direct allocation (a stray
// cudaMalloc would fragment the pool or exceed its reservation), and
// long-running or real-time hosts that must not allocate after start-up (an
// allocation can block on the device or fail at an arbitrary time).  For them
// this entry point keeps every piece of scratch the step needs -- the half
// spectrum, the per-plane partial sums, the stress/flag words, the twiddle and
// slot tables -- in one file-scope device array of PFDD_STATIC_SCRATCH_BYTES.
// Every GPU that loads the library holds that array until the process exits.
//
// Host code only ever sees a stand-in for the array's name, so the first call
// on each device (with that device current) looks its device address up with
// cudaGetSymbolAddress and caches it for the life of the process; that first
// call should therefore come before any stream capture, and cudaDeviceReset
// between calls is not supported (the cached address would be stale).  All
// calls share the one array and it keeps the last call's contents: the flags
// are cleared on every call, and calls whose work overlaps on the GPU
// (different streams, or different host threads on one device) race on it.
// Without h_stats the call reports neither divergence nor a timeout (the next
// call clears the flags unread).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "pfdd_b200.h"
#include "pfdd_setup.cuh"

using namespace pfdd;
using namespace pfdd::host;

static __device__ __align__(256) unsigned char g_noalloc_scratch[PFDD_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDev = 64;
std::mutex g_mu;
void *g_addr[kMaxDev];            // device address of g_noalloc_scratch per device
// Status codes are the only error channel of this entry point (it keeps no
// per-call message state); the message argument documents each exit.
pfdd_status nerr(pfdd_status code, const char * /*why*/) { return code; }

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

// digit-reversed position of each frequency (no heap use)
void positions_into(const FftPlan &p, int *pos) {
  for (int k = 0; k < p.n; ++k) {
    int rem = k, q = 0;
    for (int s = 0; s < p.nst; ++s) {
      const int d = rem % p.radix[s];
      rem /= p.radix[s];
      q += d * (p.L[s] / p.radix[s]);
    }
    pos[k] = q;
  }
}

void twiddles_into(int n, int count, double2 *out) {
  for (int m = 0; m < count; ++m) {
    const double ang = 2.0 * M_PI * (double)(m % n) / (double)n;
    out[m] = make_double2(std::cos(ang), -std::sin(ang));
  }
}

pfdd_status device_setup(int dev, void **addr) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= kMaxDev) return nerr(PFDD_EINVAL, "device ordinal out of range");
  if (g_addr[dev]) { *addr = g_addr[dev]; return PFDD_OK; }
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) return nerr(PFDD_ECUDA, "cudaGetSymbolAddress of the static scratch failed");
  g_addr[dev] = p;
  *addr = p;
  return PFDD_OK;
}

}  // namespace

extern "C" pfdd_status pfdd_gl_step_noalloc(const pfdd_instance_desc *desc, const double *d_xi_in,
                                            double *d_xi_out, double *h_stats, void *stream) {
  if (!desc || !d_xi_in || !d_xi_out) return nerr(PFDD_EINVAL, "desc, d_xi_in and d_xi_out are required");
  if (d_xi_in == d_xi_out) return nerr(PFDD_EINVAL, "d_xi_in and d_xi_out must not alias");
  const pfdd_instance_desc &d = *desc;
  const int S = d.n_slip;
  if (S < 1 || S > PFDD_MAX_SLIP) return nerr(PFDD_EINVAL, "n_slip outside 1..PFDD_MAX_SLIP");
  if (d.xo || d.site_gsfe) return nerr(PFDD_EINVAL, "no obstacle mask or per-site GSFE field in this entry point");
  if (d.core_flag == PFDD_CORE_MPEA || d.core_flag == PFDD_CORE_SINE_FIELD)
    return nerr(PFDD_EINVAL, "per-site GSFE core models are not available in this entry point");
  FftPlan px, py, pz;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (nx < 2 || ny < 2 || nz < 4 || nx > 1024 || ny > 1024 || nz > 1024 || (nx & 1) || (ny & 1) || (nz % 4) ||
      !make_plan(nx, px) || !make_plan(ny, py) || !make_zplan(nz / 2, pz))
    return nerr(PFDD_EUNSUPPORTED, "grid extents must be even, 2^a 3^b, <= 1024, nz a multiple of 4");
  const int M = nz / 2, nzh = M + 1, nzp = nzh;  // FP64 rows are whole 16-byte units
  const int F = 2 * S;                           // Re and Im fields
  const size_t N = (size_t)nx * ny * nz;
  typedef double2 C;

  // shared-memory layout of the pencil pass (as the handle path chooses it)
  const size_t ncols = (size_t)ny * nzp;
  auto fstride_for = [&](int cc) {
    const int target = (cc * 4) % 32;
    for (int pad = 0; pad < 64; ++pad)
      if ((((size_t)nx * cc + pad) * 4) % 32 == (size_t)target) return nx * cc + pad;
    return nx * cc;
  };
  auto pencil_bytes = [&](int cc) {
    return ((size_t)F * fstride_for(cc) + (size_t)nx) * sizeof(C) + 64 * sizeof(double) +
           ((size_t)nx + 2 * (size_t)cc) * sizeof(V4<double>) + 2 * (size_t)((cc + 3) & ~3) * sizeof(int) +
           (size_t)cc * S * sizeof(C);
  };
  int cc = 32;
  while (cc > 1 && (ncols % cc || pencil_bytes(cc) > 200 * 1024)) cc >>= 1;
  const size_t smem_plane = PlaneSmem<C>::bytes(ny, ny, nzp, M);
  if (ncols % cc || pencil_bytes(cc) > 227 * 1024 || smem_plane > 227 * 1024)
    return nerr(PFDD_EUNSUPPORTED, "grid too large for the shared-memory passes in FP64");

  // scratch layout
  const size_t b_spec = up256((size_t)F * nx * ny * nzp * sizeof(C));
  const size_t b_part = up256(2 * (size_t)F * nx * sizeof(double));
  const size_t b_small = up256((PFDD_MAXS + 9 + 8 + 2 + 2) * sizeof(double));
  const size_t b_tw = up256((size_t)(nx + ny + 2 * M) * sizeof(C));
  const size_t b_tab = up256((size_t)(M + nx + 2 * ny + nzp + M / 2) * sizeof(int16_t));
  const size_t need = b_spec + b_part + b_small + b_tw + b_tab;
  if (need > PFDD_STATIC_SCRATCH_BYTES)
    return nerr(PFDD_EINVAL, "grid needs more scratch than the static array holds; use pfdd_gpu_create");

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nerr(PFDD_ENODEVICE, "no current CUDA device");
  void *base = nullptr;
  pfdd_status st = device_setup(dev, &base);
  if (st != PFDD_OK) return st;
  // every call: a handle created since the last call may have set these
  // kernels' limits for its own sizes (raise_smem_limit never lowers them)
  if (raise_smem_limit(k_fwd_planes<double, 256, false>, smem_plane) != cudaSuccess ||
      raise_smem_limit(k_xpencil<double, 256>, pencil_bytes(cc)) != cudaSuccess ||
      raise_smem_limit(k_inv_update<double, 256, false>, smem_plane) != cudaSuccess)
    return nerr(PFDD_ECUDA, "raising the kernels' shared-memory limits failed");
  unsigned char *p = static_cast<unsigned char *>(base);
  C *spec = reinterpret_cast<C *>(p);
  double *partials = reinterpret_cast<double *>(p + b_spec);
  double *small = reinterpret_cast<double *>(p + b_spec + b_part);
  double *tau = small;                                   // [PFDD_MAXS]
  int *flags = reinterpret_cast<int *>(small + PFDD_MAXS + 9);  // stop, bad, steps, timeout
  double *stats = small + PFDD_MAXS + 9 + 8;            // xinorm, xiave
  double *an = small + PFDD_MAXS + 9 + 8 + 2;           // core model 6: An' pi, An'
  C *tw = reinterpret_cast<C *>(p + b_spec + b_part + b_small);
  int16_t *tab = reinterpret_cast<int16_t *>(p + b_spec + b_part + b_small + b_tw);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

  // host-side constants (stack buffers only)
  double2 htw[2 * 1024 + 1024];
  twiddles_into(nx, nx, htw);
  twiddles_into(ny, ny, htw + nx);
  twiddles_into(M, M, htw + nx + ny);
  twiddles_into(nz, M, htw + nx + ny + M);
  int pos[1024];
  int16_t htab[512 + 1024 + 1024 + 513 + 1024 + 256];
  memset(htab, 0, sizeof htab);
  int16_t *t_posM = htab, *t_kx = t_posM + M, *t_ky = t_kx + nx, *t_kz = t_ky + ny;
  positions_into(pz, pos);
  for (int k = 0; k < M; ++k) { t_posM[k] = (int16_t)pos[k]; t_kz[pos[k]] = (int16_t)k; }
  int16_t *t_kord = t_kz + nzp + ny;
  unpack_order(pos, M, t_kord);
  t_kz[M] = (int16_t)M;
  positions_into(px, pos);
  for (int k = 0; k < nx; ++k) t_kx[pos[k]] = (int16_t)k;
  const int sx_n = pos[nx / 2];
  positions_into(py, pos);
  for (int k = 0; k < ny; ++k) t_ky[pos[k]] = (int16_t)k;
  const int sy_n = pos[ny / 2];
  int16_t *t_neg = t_kz + nzp;
  neg_slots(ny, false, pos, t_neg);

  Green green;
  build_green(d, green);
  Core core;
  if (!build_core(d, core)) return nerr(PFDD_EUNSUPPORTED, "core model not supported");
  StressArgs sa;
  build_stress(d, sa);
  if (d.non_schmid && S > 3) return nerr(PFDD_EINVAL, "non-Schmid stress needs n_slip <= 3");
  // tau (Schmid or non-Schmid) and the core model 6 amplitude at the
  // descriptor's stress state
  double htau[PFDD_MAXS], han[2];
  resolve_state_host(sa, d.sigma, htau, han);

  cudaError_t e = cudaSuccess;
  e = cudaMemcpyAsync(tw, htw, (size_t)(nx + ny + 2 * M) * sizeof(C), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(tab, htab, (size_t)(M + nx + 2 * ny + nzp + M / 2) * sizeof(int16_t), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tau, htau, S * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(an, han, sizeof han, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, 8 * sizeof(int), s);
  if (e != cudaSuccess) return nerr(PFDD_ECUDA, cudaGetErrorString(e));

  const C *tw_x = tw, *tw_y = tw + nx, *tw_z = tw + nx + ny, *tw_r = tw + nx + ny + M;
  PlaneArgs pa;
  pa.py = py; pa.pz = pz;
  pa.nx = nx; pa.ny = ny; pa.nz = nz; pa.nzh = nzh; pa.nzp = nzp; pa.nzs = nzp; pa.M = M;
  pa.S = S; pa.F = F;
  pa.zfused = 1;
  pa.tw_y = tw_y; pa.tw_z = tw_z; pa.tw_r = tw_r;
  pa.posM = t_posM - htab + tab;
  pa.negy = t_neg - htab + tab;
  pa.kord = t_kord - htab + tab;
  set_plane_divisors<double>(pa, ny);
  PencilArgs pe;
  pe = PencilArgs{};
  pe.px = px;
  pe.nx = nx; pe.ny = ny; pe.nz = nz; pe.nzh = nzh; pe.nzp = nzp; pe.M = M;
  pe.S = S; pe.F = F; pe.imag = IMAG_FULL;
  pe.ncols = (int)ncols;
  pe.ccols = cc;
  pe.tw_x = tw_x;
  pe.kx_of = tab + (t_kx - htab); pe.ky_of = tab + (t_ky - htab); pe.kz_of = tab + (t_kz - htab);
  pe.mode = PASS_STEP;
  pe.fstride = fstride_for(cc);
  pe.sx_n = sx_n; pe.sy_n = sy_n;
  pe.cd = d.cd_dt;
  pe.g = green;
  set_pencil_divisors<double>(pe);
  UpdateArgs ua;
  memset(&ua, 0, sizeof ua);
  ua.nx = nx; ua.ny = ny; ua.nz = nz; ua.nzh = nzh; ua.nzp = nzp; ua.S = S; ua.F = F;
  ua.cd = d.cd_dt;
  ua.invN = 1.0 / (double)N;
  ua.core = core;
  ua.tau = tau;
  ua.site = d.core_flag == PFDD_CORE_USFE_ANGLE ? an : nullptr;
  ua.stop = flags;
  ua.err = flags + 3;
  ua.mode = PASS_STEP;

  const int planes = F * nx;
  k_fwd_planes<double, 256, false><<<planes, 256, smem_plane, s>>>(d_xi_in, spec, pa, flags, flags + 3);
  k_xpencil<double, 256><<<(int)(ncols / cc), 256, pencil_bytes(cc), s>>>(spec, pe, flags);
  k_inv_update<double, 256, false><<<planes, 256, smem_plane, s>>>(spec, d_xi_in, d_xi_out, pa, ua, partials);
  k_finalize<<<1, 256, 0, s>>>(partials, planes, stats, 0, 0.0, flags, flags + 1, flags + 2, nullptr, 0, 0.0);
  e = cudaGetLastError();
  if (e != cudaSuccess) return nerr(PFDD_ECUDA, cudaGetErrorString(e));
  if (h_stats) {
    double out[2];
    int fl[4];
    e = cudaMemcpyAsync(out, stats, sizeof out, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fl, flags, sizeof fl, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return nerr(PFDD_ECUDA, cudaGetErrorString(e));
    if (fl[3]) return nerr(PFDD_ETIMEOUT, "a bounded device wait ran out");
    if (fl[1]) return nerr(PFDD_EDIVERGED, "non-finite order parameter");
    h_stats[0] = out[0];
    h_stats[1] = out[1];
  }
  return PFDD_OK;
}
