// Hot-path kernels of one Ginzburg-Landau iteration (sm_100a).
//
// One GL iteration of the reference (solve_GL.cpp:92-124) on real fields
// (Re xi and, when carried, Im xi) becomes three passes over HBM:
//   P1 k_fwd_planes   per (field, x-plane): z real-to-complex FFT (half-length
//                     packing) + y FFT, in shared memory   -> half spectrum
//   P2 k_xpencil      per tile of (ky, kz) columns, all fields: x FFT, the
//                     per-k Green's contraction of internal_energy
//                     (fft_fftw_slab.cpp:1670-1695) with B(k) regenerated from
//                     k in registers, inverse x FFT          -> elastic spectrum
//   P3 k_inv_update   per (field, x-plane): inverse y FFT + z complex-to-real,
//                     fused with the GSFE core force (core_energy_*), the
//                     applied stress and the explicit Euler update with the
//                     obstacle mask (update_order_parameter,
//                     fft_fftw_slab.cpp:1746-1790), plus FP64 partial sums of
//                     |dxi|^2 and sum Re xi
// followed by a one-block FP64 compensated reduction (k_finalize).
//
// Spectrum layout: spec[f][x][sy][sz] with sy, sz the digit-reversed slots of
// ky and kz (z slot M = nz/2 holds the Nyquist column); P2 additionally
// permutes kx inside shared memory only.  Frequencies are recovered through
// slot tables, so no transform ever reorders data.
//
// DC / Nyquist packing: after the z real-to-complex transform the kz = 0 and
// kz = nz/2 columns of a plane are both real, so the y transforms carry them
// as one complex column Z = Y0 + i YM in slot 0 and run over M = nz/2 columns
// (a multiple of the warp width) instead of nz/2 + 1.  P1 splits Z back into
// Y0[ky] = (Z[ky] + conj Z[-ky]) / 2 and YM[ky] = (Z[ky] - conj Z[-ky]) / (2i)
// before storing (the spectrum layout keeps the Nyquist column at slot M);
// P3 packs Y0 + i YM before its inverse y transform, which then returns the
// two real columns as the real and imaginary parts of slot 0.
//
// Split planes (SPLIT = true): P1 and P3 can run each (field, x) plane on a
// cluster of two CTAs, CTA rank r holding rows [r ny/2, (r+1) ny/2) in its
// own shared memory; the first radix-2 stage of the y transform (rows y and
// y + ny/2) goes through distributed shared memory and the remaining
// ny/2-point stages are local.  Rank r then holds ky = r + 2 k' at the slots
// of the ny/2-point plan, which the host's ky slot table encodes.
#pragma once
#include <cooperative_groups.h>
#include <cstddef>

#include <type_traits>

#include "pfdd_fft.cuh"

#define PFDD_MAXS 12
#define PFDD_PI_T 3.14159265358979323846

namespace pfdd {

// Largest FFT radix a kernel with NT threads compiles (bounds registers:
// 1024-thread blocks must fit 64 registers per thread).
template <int NT> struct MaxRadix { static constexpr int value = NT >= 1024 ? 8 : 16; };

// Resident CTAs per SM a plane kernel is compiled for (register cap): FP32
// split planes (half a plane of shared memory each) fit three to an SM; FP64
// planes are held to 128 registers so that small planes run two to an SM.
#ifndef PFDD_SPLIT_MINB_F32
#define PFDD_SPLIT_MINB_F32 3
#endif
#ifndef PFDD_PLANE_MINB_F64
#define PFDD_PLANE_MINB_F64 1
#endif
template <typename T, bool SPLIT> struct PlaneMinBlocks {
  static constexpr int value = sizeof(T) == 4 ? (SPLIT ? PFDD_SPLIT_MINB_F32 : 1) : PFDD_PLANE_MINB_F64;
};
#ifndef PFDD_PENCIL_MINB_F32
#define PFDD_PENCIL_MINB_F32 2
#endif
// 1: with a run-time slip count the x-pencil contraction reads its constants
// from a shared-memory stage as vectors (0: scalar constant-bank loads)
#ifndef PFDD_PENCIL_SMEM_CONST
#define PFDD_PENCIL_SMEM_CONST 0
#endif
template <typename T> struct PencilMinBlocks {
  static constexpr int value = sizeof(T) == 4 ? PFDD_PENCIL_MINB_F32 : 1;
};

// Per-instance constants of the contraction and the update (FP64 on the host).
// Each table is kept in FP64 (set-up, FP64 path) and rounded once to FP32
// (FP32 path), so the kernels never convert constants in their inner loops.
template <typename T> struct GreenT {
  T four[3][3];
  T sig[PFDD_MAXS][6];    // sigma^a = C : eps^a  (xx yy zz xy xz yz), to build Sig = sum_b Y_b sigma^b
  T sigo[PFDD_MAXS][6];   // sigma^a / mu with off-diagonals counted twice (contracts the symmetric T)
  T epso[PFDD_MAXS][6];   // eps^a / mu: xx yy zz, xy+yx, xz+zx, yz+zy (contracts Sig)
  T c2;                   // 1 / (2 C44), Green's function prefactor, fft_fftw_slab.cpp:597
  T c1nu;                 // 1 / (1 - nu) (Voigt nu)
  // tf = 1 when sigo[a] = lam o epso[a] for every system (glide systems,
  // b . n = 0, so sigma^a = C44 (eps^a + eps^a^T)): lam = 2 C44 on the
  // diagonal, C44 off it, and each output off the Nyquist planes is the one
  // contraction eps^a : Z with Z = Sig + lam o Tq (green_z)
  T lam[6];
  int tf;
};
struct Green {
  double four[3][3];
  double sig[PFDD_MAXS][6];   // sigma^a = C : eps^a  (xx yy zz xy xz yz)
  double eps[PFDD_MAXS][6];   // eps^a contracted with a symmetric tensor: xx yy zz, xy+yx, xz+zx, yz+zy
  double inv_mu;              // 1 / mu (Voigt), fft_fftw_slab.cpp:628
  double c2;                  // 1 / (2 C44), Green's function prefactor, fft_fftw_slab.cpp:597
  double c1nu;                // 1 / (1 - nu) (Voigt nu)
  GreenT<double> d;
  GreenT<float> f;
};
template <typename T> __device__ __forceinline__ const GreenT<T> &green_t(const Green &g);
template <> __device__ __forceinline__ const GreenT<double> &green_t<double>(const Green &g) { return g.d; }
template <> __device__ __forceinline__ const GreenT<float> &green_t<float>(const Green &g) { return g.f; }

struct Core {
  int flag;
  double k[12];               // scaled constants, see core_derivative
  float kf[12];               // the same, rounded once for the FP32 path
  // core model 5 (the angle between the line direction and b): grid, `four`
  // and the slip normals / Burgers vectors
  int nx, ny, nz;
  double four[3][3];
  double xn[PFDD_MAXS][3], xb[PFDD_MAXS][3];
};
template <typename T> __device__ __forceinline__ T core_k(const Core &c, int i);
template <> __device__ __forceinline__ double core_k<double>(const Core &c, int i) { return c.k[i]; }
template <> __device__ __forceinline__ float core_k<float>(const Core &c, int i) { return c.kf[i]; }

// IMAG_NONE: Re xi only, B averaged over k and index -k (not reference-exact)
// IMAG_FULL: Im xi carried as a second real field through every pass
// IMAG_NYQ:  Im xi carried as its spectrum on the Nyquist planes only, where
//            it lives when no obstacle mask is set (updated inside P2)
enum { IMAG_NONE = 0, IMAG_FULL = 1, IMAG_NYQ = 2 };
enum { PASS_STEP = 0, PASS_SYNTH = 1, PASS_ADJOINT = 2, PASS_ENERGY = 3 };

struct PlaneArgs {
  FftPlan py, pz;
  int nx, ny, nz, nzh, nzp, M;   // nzp: complex entries per stored spectrum row (>= nzh, 16-byte rows)
  int nzs;                       // complex entries per shared-memory row (>= nzp, chosen against bank conflicts)
  int S, F;                   // slip systems; fields in flight (S, or 2S with Im xi)
  const void *tw_y, *tw_z, *tw_r;   // W_ny^m, W_M^m, W_nz^k tables in compute precision
  const int16_t *posM;        // position of z-frequency k (< M) after the M-point transform
  const int16_t *kord;        // k = 1..M/2 ordered by posM[k]: real/complex (un)packing pairs in slot order
  const int16_t *negy;        // slot of -ky for each local y slot (a split plane's rank r at r * rows)
  // divisors built on the host: rows per CTA (ny, or ny/2 when split),
  // nz / vector width, M, M/2 (real-to-complex pairs per row)
  FastDiv fd_rows, fd_nvec, fd_m, fd_mh;
  int zfused;                 // 1: update and adjoint passes may take the register-resident z passes
};

struct PencilArgs {
  FftPlan px;
  int nx, ny, nz, nzh, nzp, M;
  int S, F, imag;
  int ncols;                  // ny * nzp
  int ccols;                  // columns per CTA
  const void *tw_x;
  const int16_t *kx_of, *ky_of, *kz_of;   // frequency index of each slot (kz_of has nzp entries)
  int mode;                   // PASS_STEP or PASS_SYNTH (rebuild Im xi from the Nyquist spectrum)
  int fstride;                // shared-memory stride between fields (complex), bank-conflict padded
  // Nyquist spectrum of Im xi (IMAG_NYQ): kz = nz/2 plane [S][nx][ny], ky = ny/2
  // plane [S][nx][M], kx = nx/2 plane [S][ny][M] (slot coordinates)
  void *aux;
  int sx_n, sy_n;             // slots of kx = nx/2 and ky = ny/2
  double cd;                  // CD * timestep
  double *partials;           // per-CTA sum of |d Im xi|^2 * N (Parseval weight), or null
  // divisors built on the host: F * ccols, ccols, nzp, 16-byte chunks per
  // (field, x) row of a tile, nx
  FastDiv fd_fcc, fd_cc, fd_nzp, fd_cpr, fd_nx;
  FastDiv fd_6cc;             // strain diagnostics: 6 * ccols (conductivity pencil: 4 * ccols)
  double inv2mu;              // strain diagnostics: 1 / (2 mu), Voigt mu (Fmatrix, fft_fftw_slab.cpp:657)
  Green g;
};

struct UpdateArgs {
  int nx, ny, nz, nzh, nzp, S, F;
  int mode;                   // PASS_STEP: GL update; PASS_SYNTH: xout = IFFT(spec)/N;
                              // PASS_ADJOINT: adjoint update of lambda (xin) at forward state xfwd
  const void *xfwd;           // PASS_ADJOINT: Re xi_n [S][N] (compute precision)
  double *gpart;              // PASS_ADJOINT: per-plane {sum lam df'/d p0, sum lam df'/d p1, sum lam}
  double cd;                  // CD * timestep
  double invN;
  Core core;
  const double *tau;          // [S] device, FP64
  const uint8_t *mask;        // [S*N] or null
  const void *site;           // [S*N] per-site GSFE field (compute precision) or null
  const int *stop;            // device flag: skip the step when nonzero
  int *err;                   // device flag: a bounded wait ran out
};

// Per-instance device pointers of a batched group: the batched kernel entries
// take a table of these and handle instance blockIdx.y, so one launch covers
// every instance of a group (same grid shape and constants, own state, stress,
// mask and per-site GSFE).  The flags word block is the instance's control
// state on the device: [0] stop (tolerance reached), [1] non-finite, [2]
// steps done (also the stats record index), [3] a bounded wait ran out,
// [4] which xi buffer holds the current state.  Keeping the buffer parity on
// the device makes a step's launches independent of how many earlier steps
// were skipped, so they can be replayed from a CUDA graph.
struct InstPtrs {
  void *xi[2];
  void *spec;
  void *aux;
  double *ppart;       // x-pencil partial sums (Nyquist carrier) or null
  double *partials;    // plane partial sums
  double *tau;         // [S]
  double *sigma;       // [9] current stress, [9] increment per stress state
  int *flags;
  double *stats;       // {xinorm, xiave} per step
  int stats_cap;
  const uint8_t *mask;
  const void *site;
  double *an;          // core model 6 amplitude slots (resolve_state), or null
};

// ------------------------------------------------------------ small helpers
template <typename T> struct __align__(16) V4 { T x, y, z, w; };
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
// correctly rounded reciprocal
__device__ __forceinline__ float recip_t(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip_t(double x) { return 1.0 / x; }

// sin(pi y) and cos(pi y) of the FP32 path (this project's polynomials, not
// a library routine): y = n/2 + t with n = rint(2y), |t| <= 1/4, then
// sin(pi t) = t S(t^2) and cos(pi t) = C(t^2) with S of degree 3 and C of
// degree 4 (least-squares fits, in FP64, of sin(pi t)/t and cos(pi t) over
// 2000 Chebyshev nodes of 0 < t <= 1/4, weighted for relative error and
// rounded to FP32), and the quadrant n mod 4 rotates (sin, cos).  Error
// within 2 ulp of sin(pi y), cos(pi y) for |y| < 2^22
// (tests/test_sincospi_cpu.py).
__device__ __forceinline__ void sincospi_poly(float y, float *s, float *c) {
  const float n = rintf(2.0f * y);
  const float t = __fmaf_rn(n, -0.5f, y);   // exact
  const float u = t * t;
  float ps = __fmaf_rn(u, -0.5890104174613953f, 2.5497608184814453f);
  ps = __fmaf_rn(u, ps, -5.167707443237305f);
  ps = __fmaf_rn(u, ps, 3.1415927410125732f);
  const float sv = t * ps;
  float pc = __fmaf_rn(u, 0.23126046359539032f, -1.335035800933838f);
  pc = __fmaf_rn(u, pc, 4.058706760406494f);
  pc = __fmaf_rn(u, pc, -4.934802055358887f);
  const float cv = __fmaf_rn(u, pc, 1.0f);
  const int q = (int)n & 3;
  float ss = (q & 1) ? cv : sv, cs = (q & 1) ? sv : cv;
  if (q & 2) ss = -ss;
  if ((q + 1) & 2) cs = -cs;
  *s = ss;
  *c = cs;
}

template <typename T> __device__ __forceinline__ void sincospi_t(T x, T *s, T *c);
template <> __device__ __forceinline__ void sincospi_t<double>(double x, double *s, double *c) { sincospi(x, s, c); }
template <> __device__ __forceinline__ void sincospi_t<float>(float x, float *s, float *c) { sincospi_poly(x, s, c); }
template <typename T> __device__ __forceinline__ T sinpi_t(T x);
template <> __device__ __forceinline__ double sinpi_t<double>(double x) { return sinpi(x); }
template <> __device__ __forceinline__ float sinpi_t<float>(float x) {
  float s, c;
  sincospi_poly(x, &s, &c);
  return s;
}
template <typename T> __device__ __forceinline__ T cospi_t(T x);
template <> __device__ __forceinline__ double cospi_t<double>(double x) { return cospi(x); }
template <> __device__ __forceinline__ float cospi_t<float>(float x) {
  float s, c;
  sincospi_poly(x, &s, &c);
  return c;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-reduce two doubles into out[0..1] (thread 0 writes). smem: 2*32 doubles.
__device__ __forceinline__ void block_sum2(double a, double b, double *scratch, double *out) {
  a = warp_sum(a);
  b = warp_sum(b);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) { scratch[wid] = a; scratch[32 + wid] = b; }
  __syncthreads();
  if (wid == 0) {
    a = lane < nw ? scratch[lane] : 0.0;
    b = lane < nw ? scratch[32 + lane] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) { out[0] = a; out[1] = b; }
  }
}

// Block-reduce NV doubles; warp 0 ends with the totals (thread 0 uses them).
// scratch: NV*32 doubles.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double *scratch) {
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) scratch[q * 32 + wid] = v[q];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(lane < nw ? scratch[q * 32 + lane] : 0.0);
  }
}

// Sum of NV doubles over the CTA (SPLIT: over both CTAs of the plane's
// cluster, rank 1 handing its totals to rank 0 through distributed shared
// memory) written to out[0..NV-1] by one thread.  scratch: NV*32 + NV doubles.
// Every thread of both CTAs must call it.
// ACCUM: added to out[] instead of stored (a running sum over launches; one
// CTA or CTA pair owns each plane's out[], so no other thread writes it).
template <bool SPLIT, int NV, bool ACCUM = false>
__device__ __forceinline__ void plane_sum(double (&v)[NV], double *scratch, double *out) {
  block_reduce<NV>(v, scratch);
  if constexpr (!SPLIT) {
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < NV; ++q) out[q] = ACCUM ? out[q] + v[q] : v[q];
    }
  } else {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    double *slot = scratch + NV * 32;
    if (rank == 1 && threadIdx.x == 0) {
      double *peer = cl.map_shared_rank(slot, 0);
#pragma unroll
      for (int q = 0; q < NV; ++q) peer[q] = v[q];
    }
    cl.sync();
    if (rank == 0 && threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < NV; ++q) out[q] = ACCUM ? out[q] + (v[q] + slot[q]) : v[q] + slot[q];
    }
  }
}

// The same sums written without a cluster barrier (whose release fence would
// wait for the plane pass's global stores): slot `plane`, or for a split
// plane each CTA its own slot 2 plane + rank, which the reduction kernel adds
// in order.  out: NV doubles per slot.
template <bool SPLIT, int NV>
__device__ __forceinline__ void plane_sum_slots(double (&v)[NV], double *scratch, double *out, size_t plane) {
  block_reduce<NV>(v, scratch);
  if (threadIdx.x == 0) {
    size_t slot = plane;
    if constexpr (SPLIT) slot = 2 * plane + cooperative_groups::this_cluster().block_rank();
#pragma unroll
    for (int q = 0; q < NV; ++q) out[NV * slot + q] = v[q];
  }
}

// The cross-CTA radix-2 stage of a split plane, over the nzh slot columns of
// the ny/2 local rows.  Forward (decimation in frequency): lo = a + b,
// hi = (a - b) W_ny^y with a, b rows y and y + ny/2; inverse (decimation in
// time, unnormalised): lo = E + O conj(W_ny^y), hi = E - O conj(W_ny^y).  Each
// pair (y, c) is read and written by one thread of one CTA (rank 0 takes the
// first half of the pairs), so no result overwrites a value still to be read;
// the cluster barriers before and after order it against both CTAs' own
// passes.  twx2: W_ny^y, y < ny/2.
template <bool INV, typename C>
__device__ __forceinline__ void cross_stage(C *buf, const C *__restrict__ twx2, int nyh, const FastDiv &dz,
                                            int nzs) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank();
  C *peer = cl.map_shared_rank(buf, rank ^ 1u);
  C *lo = rank == 0 ? buf : peer;
  C *hi = rank == 0 ? peer : buf;
  const int nzh = (int)dz.d;
  const int total = nyh * nzh;
  const int begin = rank == 0 ? 0 : total / 2, end = rank == 0 ? total / 2 : total;
  cl.sync();
#ifndef PFDD_CROSS_U
#define PFDD_CROSS_U 4
#endif
  constexpr int U = PFDD_CROSS_U;   // pairs in flight per thread
  for (int i0 = begin + threadIdx.x; i0 < end; i0 += U * blockDim.x) {
    C a[U], b[U], w[U];
    size_t o[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
      const int i = i0 + q * blockDim.x;
      const int ii = i < end ? i : begin;
      const int y = dz.div(ii), c = ii - y * nzh;
      o[q] = (size_t)y * nzs + c;
      a[q] = lo[o[q]];
      b[q] = hi[o[q]];
      w[q] = twx2[y];
    }
#pragma unroll
    for (int q = 0; q < U; ++q) {
      if (i0 + q * blockDim.x >= end) continue;
      if (!INV) {
        lo[o[q]] = cadd(a[q], b[q]);
        hi[o[q]] = cmul(csub(a[q], b[q]), w[q]);
      } else {
        const C t = cmulc(b[q], w[q]);
        lo[o[q]] = cadd(a[q], t);
        hi[o[q]] = csub(a[q], t);
      }
    }
  }
  cl.sync();
}

template <typename C>
__device__ __forceinline__ void load_table(C *dst, const void *src, int n) {
  const C *s = reinterpret_cast<const C *>(src);
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = s[i];
}

// ------------------------------------------------------------ P1
// Shared memory of a plane kernel: `rows` complex rows of stride nzs (ny, or
// ny/2 for a split plane), then the y, z and real-to-complex twiddle tables,
// the z position table, one mbarrier and the reduction scratch.  The y table
// has ny entries: W_ny^m (m < ny), or for a split plane W_ny^m (m < ny/2)
// followed by the W_{ny/2}^m of the local stages.
constexpr int kPlaneRed = 136;   // doubles of reduction scratch (4 sums)

template <typename C> struct PlaneSmem {
  C *buf, *twy, *twz, *twr;
  int *pos, *kord;
  uint64_t *bar;
  double *red;
  __device__ PlaneSmem(unsigned char *raw, const PlaneArgs &a, int rows) {
    buf = reinterpret_cast<C *>(raw);
    twy = buf + (size_t)rows * a.nzs;
    twz = twy + a.ny;
    twr = twz + a.M;
    pos = reinterpret_cast<int *>(twr + a.M);
    kord = pos + ((a.M + 1) & ~1);
    bar = reinterpret_cast<uint64_t *>(kord + ((a.M / 2 + 1) & ~1));
    red = reinterpret_cast<double *>(bar + 1);
  }
  static size_t bytes(int rows, int ny, int nzs, int M) {
    return ((size_t)rows * nzs + ny + 2 * (size_t)M) * sizeof(C) + (size_t)((M + 1) & ~1) * 4 +
           (size_t)((M / 2 + 1) & ~1) * 4 + 8 + kPlaneRed * 8;
  }
};

template <typename C>
__device__ __forceinline__ void load_plane_tables(const PlaneSmem<C> &sm, const PlaneArgs &a) {
  load_table(sm.twy, a.tw_y, a.ny);
  load_table(sm.twz, a.tw_z, a.M);
  load_table(sm.twr, a.tw_r, a.M);
  for (int i = threadIdx.x; i < a.M; i += blockDim.x) sm.pos[i] = a.posM[i];
  for (int i = threadIdx.x; i < a.M / 2; i += blockDim.x) sm.kord[i] = a.kord[i];
}

// plane index and first row of this CTA (grid.x = planes, or 2 planes for SPLIT)
template <bool SPLIT> __device__ __forceinline__ size_t plane_of_block() {
  return SPLIT ? (size_t)(blockIdx.x >> 1) : (size_t)blockIdx.x;
}
template <bool SPLIT> __device__ __forceinline__ int row0_of_block(int ny) {
  if constexpr (SPLIT) return (int)cooperative_groups::this_cluster().block_rank() * (ny / 2);
  return 0;
}

template <typename T, int NT, bool SPLIT>
__device__ __forceinline__ void fwd_planes_compute(const PlaneSmem<cx<T>> &sm, const PlaneArgs &a,
                                                   cx<T> *__restrict__ spec, size_t plane, int rows, int row0,
                                                   bool ok);

template <typename T, int NT, bool SPLIT>
__device__ __forceinline__ void fwd_planes_body(const T *__restrict__ xi, cx<T> *__restrict__ spec,
                                                const PlaneArgs &a, int *err, size_t plane) {
  using C = cx<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int ny = a.ny, nz = a.nz, nzs = a.nzs;
  const int rows = SPLIT ? ny / 2 : ny;
  const int row0 = row0_of_block<SPLIT>(ny);
  const PlaneSmem<C> sm(smem_raw, a, rows);
  const int stall = stall_switch(err);
  if (threadIdx.x == 0) mbar_init(sm.bar, 1 + stall);
  __syncthreads();
  // rows of the real plane -> shared rows of stride 2*nzs reals (bulk copies)
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) mbar_expect_tx(sm.bar, (uint32_t)(rows * nz * sizeof(T)));
    __syncwarp();
    const T *src = xi + (plane * (size_t)ny + row0) * nz;
    T *bufr = reinterpret_cast<T *>(sm.buf);
    for (int y = threadIdx.x; y < rows; y += 32)
      bulk_g2s(bufr + (size_t)y * 2 * nzs, src + (size_t)y * nz, (uint32_t)(nz * sizeof(T)), sm.bar);
  }
  load_plane_tables(sm, a);
  const bool ok = plane_wait(sm.bar, stall, err);
  // after a timeout a split CTA carries on without storing: its peer waits at the cluster barriers
  if (!ok && !SPLIT) return;
  fwd_planes_compute<T, NT, SPLIT>(sm, a, spec, plane, rows, row0, ok);
}

template <typename T, int NT, bool SPLIT>
__device__ __forceinline__ void fwd_planes_tail(const PlaneSmem<cx<T>> &sm, const PlaneArgs &a,
                                                cx<T> *__restrict__ spec, size_t plane, int rows, int row0,
                                                bool ok);
template <typename T, int NT>
__device__ __forceinline__ void fwd_planes_z(const PlaneSmem<cx<T>> &sm, const PlaneArgs &a, int rows);

// The forward part of P1 on the real rows already in shared memory (row
// stride 2*nzs reals): z real-to-complex, y, DC/Nyquist split, bulk store of
// the half-spectrum rows.  `ok` false: compute (a split peer waits at the
// cluster barriers) but store nothing.  Every thread of the CTA calls it.
template <typename T, int NT, bool SPLIT>
__device__ __forceinline__ void fwd_planes_compute(const PlaneSmem<cx<T>> &sm, const PlaneArgs &a,
                                                   cx<T> *__restrict__ spec, size_t plane, int rows, int row0,
                                                   bool ok) {
  fwd_planes_z<T, NT>(sm, a, rows);
  fwd_planes_tail<T, NT, SPLIT>(sm, a, spec, plane, rows, row0, ok);
}

// The z side of the forward part: the M-point transforms of the packed real
// rows and the real-to-complex unpacking (no barrier at the end).
template <typename T, int NT>
__device__ __forceinline__ void fwd_planes_z(const PlaneSmem<cx<T>> &sm, const PlaneArgs &a, int rows) {
  using C = cx<T>;
  const int nzh = a.nzh, nzp = a.nzp, nzs = a.nzs, M = a.M;
  C *buf = sm.buf;
  const C *twr = sm.twr;
  const int *pos = sm.pos;

  // z: M-point complex transform of the packed rows
  Batch gz{rows, rows, nzs, 0, 1, false, a.fd_rows, a.fd_rows};
  fft_forward<MaxRadix<NT>::value, GeomRows>(buf, sm.twz, a.pz, gz);

  // real-to-complex unpacking, pairs (k, M-k); X[M] rides in slot 0 (see the packing note)
  // k = 0 and the row padding, one row per thread: X[0] = z0.x + z0.y and
  // X[M] = z0.x - z0.y are real, packed as X[0] + i X[M]
  for (int y = threadIdx.x; y < rows; y += blockDim.x) {
    C *row = buf + (size_t)y * nzs;
    C z0 = row[pos[0]];
    row[pos[0]] = mk<C>(z0.x + z0.y, z0.x - z0.y);
    for (int q = nzh; q < nzp; ++q) row[q] = mk<C>((T)0, (T)0);
  }
  // pairs (k, M-k), k = 1..M/2 taken in slot order (few bank conflicts)
  const int mh = M / 2;
  const int *kord = sm.kord;
  for (int w = threadIdx.x; w < rows * mh; w += blockDim.x) {
    const int y = a.fd_mh.div(w), k = kord[w - y * mh];
    C *row = buf + (size_t)y * nzs;
    {
      const int pk = pos[k], pm = pos[M - k];
      C zk = row[pk], zm = row[pm];
      // E = (Zk + conj Zm)/2, O = (Zk - conj Zm)/(2i), X[k] = E + W^k O, X[M-k] = conj(E - W^k O)
      C e = mk<C>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y));
      C o = mk<C>((T)0.5 * (zk.y + zm.y), (T)-0.5 * (zk.x - zm.x));
      C wo = cmul(twr[k], o);
      row[pk] = cadd(e, wo);
      if (pm != pk) row[pm] = cconj(csub(e, wo));
    }
  }
}

// The y side of the forward part, after the z transforms and the
// real-to-complex unpacking of every row: the cross-CTA stage (SPLIT) or a
// barrier, the y transforms, the DC/Nyquist split and the bulk store.
template <typename T, int NT, bool SPLIT>
__device__ __forceinline__ void fwd_planes_tail(const PlaneSmem<cx<T>> &sm, const PlaneArgs &a,
                                                cx<T> *__restrict__ spec, size_t plane, int rows, int row0,
                                                bool ok) {
  using C = cx<T>;
  const int ny = a.ny, nzp = a.nzp, nzs = a.nzs, M = a.M;
  C *buf = sm.buf;
  if constexpr (SPLIT) cross_stage<false>(buf, sm.twy, rows, a.fd_m, nzs);
  else __syncthreads();

  // y: (ny or ny/2)-point transforms over the M slot columns (Nyquist packed in slot 0)
  Batch gy{M, M, 1, 0, nzs, true, a.fd_m, a.fd_m};
  fft_forward<MaxRadix<NT>::value, GeomCols>(buf, SPLIT ? sm.twy + rows : sm.twy, a.py, gy);

  // split slot 0 into the kz = 0 (slot 0) and kz = nz/2 (slot M) spectra; the
  // partner -ky of a local slot lies in the same CTA (ky and -ky have equal parity)
  {
    const int16_t *neg = a.negy + row0;
    for (int y = threadIdx.x; y < rows; y += blockDim.x) {
      const int t = neg[y];
      if (t < y) continue;   // the pair is handled by the thread of its smaller slot
      C *ps = buf + (size_t)y * nzs, *pt = buf + (size_t)t * nzs;
      const C zs = ps[0], zt = pt[0];
      const C y0 = mk<C>((T)0.5 * (zs.x + zt.x), (T)0.5 * (zs.y - zt.y));
      const C ym = mk<C>((T)0.5 * (zs.y + zt.y), (T)-0.5 * (zs.x - zt.x));
      ps[0] = y0;
      ps[M] = ym;
      if (t != y) {
        pt[0] = cconj(y0);
        pt[M] = cconj(ym);
      }
    }
  }

  // rows -> spectrum rows of nzp entries (bulk stores)
  fence_proxy_async();
  __syncthreads();
  if (!ok) return;
  C *dst = spec + (plane * (size_t)ny + row0) * nzp;
  if (nzs == nzp) {
    if (threadIdx.x == 0) {  // rows are contiguous in both: one bulk copy
      bulk_s2g(dst, buf, (uint32_t)((size_t)rows * nzp * sizeof(C)));
      bulk_commit();
      bulk_wait_all();
    }
  } else if (threadIdx.x < 32) {
    for (int y = threadIdx.x; y < rows; y += 32)
      bulk_s2g(dst + (size_t)y * nzp, buf + (size_t)y * nzs, (uint32_t)(nzp * sizeof(C)));
    bulk_commit();
    bulk_wait_all();
  }
}

// grid.x = F * nx planes (SPLIT: 2 F nx CTAs in clusters of 2)
template <typename T, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, SPLIT>::value)) k_fwd_planes(const T *__restrict__ xi, cx<T> *__restrict__ spec,
                                                   PlaneArgs a, const int *__restrict__ stop, int *err) {
  if (stop && *stop) return;   // both CTAs of a cluster read the same flag
  fwd_planes_body<T, NT, SPLIT>(xi, spec, a, err, plane_of_block<SPLIT>());
}

// grid = (F * nx planes [x 2 for SPLIT], instances of the group)
template <typename T, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, SPLIT>::value)) k_fwd_planes_tab(const InstPtrs *__restrict__ tab, PlaneArgs a) {
  const InstPtrs &ip = tab[blockIdx.y];
  if (ip.flags[0]) return;
  const T *xi = static_cast<const T *>(ip.xi[ip.flags[4]]);
  fwd_planes_body<T, NT, SPLIT>(xi, static_cast<cx<T> *>(ip.spec), a, ip.flags + 3, plane_of_block<SPLIT>());
}

// ------------------------------------------------------------ B(k) operator
// out_a = sum_b B_ab(k) Y_b for complex Y, with the closed form of Bmatrix
// (fft_fftw_slab.cpp:587-629):  B_ab = (eps^a:C:eps^b - t^b.G.t^a)/mu,
// t^a = sigma^a k, G = (2 I/k^2 - k k^T/((1-nu) k^4)) / (2 C44).
// Because t^a is linear in sigma^a, with Sig = sum_b Y_b sigma^b, U = Sig k,
// V = k.U:
//   sum_b B_ab Y_b = (eps^a : Sig + sigma^a : Tq) / mu,
//   Tq = -2 sym(U k^T)/(2 C44 k^2) + V k k^T/((1-nu) 2 C44 k^4)
// so each k costs one 6-component Tq and 12 complex-real products per system.
// B(0) = 0 (A = 0 at k = 0 in the reference): green_tensor reports zero.
template <typename T, typename C>
__device__ __forceinline__ bool green_tensor(const GreenT<T> &g, const C (&sig)[6], T kx, T ky, T kz, C (&Tq)[6]) {
  const T k2 = kx * kx + ky * ky + kz * kz;
  if (!(k2 > (T)0)) return false;
  const T ik2 = recip_t(k2);
  const T g1 = (T)2 * ik2 * g.c2;
  const T g2 = ik2 * ik2 * g.c1nu * g.c2;
  // sig order: xx yy zz xy xz yz
  const C U0 = mk<C>(sig[0].x * kx + sig[3].x * ky + sig[4].x * kz, sig[0].y * kx + sig[3].y * ky + sig[4].y * kz);
  const C U1 = mk<C>(sig[3].x * kx + sig[1].x * ky + sig[5].x * kz, sig[3].y * kx + sig[1].y * ky + sig[5].y * kz);
  const C U2 = mk<C>(sig[4].x * kx + sig[5].x * ky + sig[2].x * kz, sig[4].y * kx + sig[5].y * ky + sig[2].y * kz);
  const C V = mk<C>(kx * U0.x + ky * U1.x + kz * U2.x, kx * U0.y + ky * U1.y + kz * U2.y);
  const C gv = mk<C>(g2 * V.x, g2 * V.y);
  // diagonal: -g1 U_i k_i + g2 V k_i^2 ; off-diagonal pair sums: -g1 (U_i k_j + U_j k_i) + 2 g2 V k_i k_j
  Tq[0] = mk<C>(-g1 * U0.x * kx + gv.x * kx * kx, -g1 * U0.y * kx + gv.y * kx * kx);
  Tq[1] = mk<C>(-g1 * U1.x * ky + gv.x * ky * ky, -g1 * U1.y * ky + gv.y * ky * ky);
  Tq[2] = mk<C>(-g1 * U2.x * kz + gv.x * kz * kz, -g1 * U2.y * kz + gv.y * kz * kz);
  const T kxy = (T)2 * kx * ky, kxz = (T)2 * kx * kz, kyz = (T)2 * ky * kz;
  Tq[3] = mk<C>(-g1 * (U0.x * ky + U1.x * kx) + gv.x * kxy, -g1 * (U0.y * ky + U1.y * kx) + gv.y * kxy);
  Tq[4] = mk<C>(-g1 * (U0.x * kz + U2.x * kx) + gv.x * kxz, -g1 * (U0.y * kz + U2.y * kx) + gv.y * kxz);
  Tq[5] = mk<C>(-g1 * (U1.x * kz + U2.x * ky) + gv.x * kyz, -g1 * (U1.y * kz + U2.y * ky) + gv.y * kyz);
  return true;
}

// (eps^a : Sig + sigma^a : Tq) / mu for system a; zero when k = 0
template <typename T, typename C>
__device__ __forceinline__ C green_out(const GreenT<T> &g, int a, const C (&sig)[6], const C (&Tq)[6], bool nz) {
  if (!nz) return mk<C>((T)0, (T)0);
  const T *e = g.epso[a];
  const T *o = g.sigo[a];
  // eps^a : Sig and sigma^a : Tq as separate chains (shorter dependences)
  T ex = (T)0, ey = (T)0, ox = (T)0, oy = (T)0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    ex = fma_t(e[q], sig[q].x, ex);
    ey = fma_t(e[q], sig[q].y, ey);
    ox = fma_t(o[q], Tq[q].x, ox);
    oy = fma_t(o[q], Tq[q].y, oy);
  }
  return mk<C>(ex + ox, ey + oy);
}

template <typename T, typename C>
__device__ __forceinline__ void green_accumulate(const GreenT<T> &g, int b, C x, C (&sig)[6]) {
  const T *s = g.sig[b];
#pragma unroll
  for (int q = 0; q < 6; ++q) { sig[q].x += s[q] * x.x; sig[q].y += s[q] * x.y; }
}

// Z = Sig + lam o Tq (zero at k = 0) for GreenT::tf, and the output
// eps^a : Z / mu of system a: 12 multiply-adds per output instead of 24
template <typename T, typename C>
__device__ __forceinline__ void green_z(const GreenT<T> &g, const C (&sig)[6], const C (&Tq)[6], bool nz, C (&Z)[6]) {
#pragma unroll
  for (int q = 0; q < 6; ++q)
    Z[q] = nz ? mk<C>(fma_t(g.lam[q], Tq[q].x, sig[q].x), fma_t(g.lam[q], Tq[q].y, sig[q].y)) : mk<C>((T)0, (T)0);
}
template <typename T, typename C>
__device__ __forceinline__ C green_out_z(const GreenT<T> &g, int a, const C (&Z)[6]) {
  const T *e = g.epso[a];
  T ex = (T)0, ey = (T)0, fx = (T)0, fy = (T)0;   // two chains
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    ex = fma_t(e[q], Z[q].x, ex);
    ey = fma_t(e[q], Z[q].y, ey);
    fx = fma_t(e[3 + q], Z[3 + q].x, fx);
    fy = fma_t(e[3 + q], Z[3 + q].y, fy);
  }
  return mk<C>(ex + fx, ey + fy);
}

// The same two operations with one system's constants read from a
// shared-memory stage as pairs (cs: sig[6] per system; co: epso[6], sigo[6]
// per system): 3 and 6 vector loads instead of 6 and 12 scalar constant loads
// when the system index is only known at run time.
template <typename T> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };
template <typename T, typename C>
__device__ __forceinline__ void green_accumulate_s(const T *__restrict__ cs, int b, C x, C (&sig)[6]) {
  using P = typename Pair<T>::type;
  const P *p = reinterpret_cast<const P *>(cs + 6 * b);
  const P a0 = p[0], a1 = p[1], a2 = p[2];
  const T v[6] = {a0.x, a0.y, a1.x, a1.y, a2.x, a2.y};
#pragma unroll
  for (int q = 0; q < 6; ++q) { sig[q].x += v[q] * x.x; sig[q].y += v[q] * x.y; }
}
template <typename T, typename C>
__device__ __forceinline__ C green_out_s(const T *__restrict__ co, int a, const C (&sig)[6], const C (&Tq)[6], bool nz) {
  if (!nz) return mk<C>((T)0, (T)0);
  using P = typename Pair<T>::type;
  const P *p = reinterpret_cast<const P *>(co + 12 * a);
  T e[6], o[6];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const P pe = p[i], po = p[3 + i];
    e[2 * i] = pe.x; e[2 * i + 1] = pe.y;
    o[2 * i] = po.x; o[2 * i + 1] = po.y;
  }
  T ex = (T)0, ey = (T)0, ox = (T)0, oy = (T)0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    ex = fma_t(e[q], sig[q].x, ex);
    ey = fma_t(e[q], sig[q].y, ey);
    ox = fma_t(o[q], Tq[q].x, ox);
    oy = fma_t(o[q], Tq[q].y, oy);
  }
  return mk<C>(ex + ox, ey + oy);
}

// frequency of index i on an axis of length n (frec, fft_fftw_slab.cpp:295-330)
template <typename T> __device__ __forceinline__ T freq_of(int i, int n) {
  return (i >= n / 2) ? (T)(i - n) / (T)n : (T)i / (T)n;
}
// frequency used by the reference at index (-i mod n): -f(i) except at n/2
template <typename T> __device__ __forceinline__ T freq_neg(int i, int n) {
  const int j = (n - i) % n;
  return freq_of<T>(j, n);
}

// ------------------------------------------------------------ P2
// grid.x = ncols / ccols tiles; dynamic smem = (F*fstride + nx) * sizeof(C) + scratch + wave-vector parts
template <typename T, typename C>
__device__ __forceinline__ size_t nyq_index(const PencilArgs &a, int f, int sx, int sy, int sz, bool &is_nyq) {
  // returns the aux slot of a Nyquist point; is_nyq false for ordinary points
  const size_t nzZ = (size_t)a.S * a.nx * a.ny, nzY = (size_t)a.S * a.nx * a.M;
  is_nyq = true;
  if (sz == a.M) return ((size_t)f * a.nx + sx) * a.ny + sy;
  if (sz > a.M) { is_nyq = false; return 0; }   // row padding
  if (sy == a.sy_n) return nzZ + ((size_t)f * a.nx + sx) * a.M + sz;
  if (sx == a.sx_n) return nzZ + nzY + ((size_t)f * a.ny + sy) * a.M + sz;
  is_nyq = false;
  return 0;
}

// SC > 0: the slip-system count is the constant SC (contraction loops
// unrolled, the per-system constants read as immediates of the parameter
// block); 0: a.S at run time.
// gt: the contraction's constant tables (green_t<T>(a.g), or one copy shared
// by the groups of a mixed-size launch); tile: this CTA's column tile.
template <typename T, int NT, int SC>
__device__ __forceinline__ void xpencil_body(cx<T> *__restrict__ spec, const PencilArgs &a, const GreenT<T> &gt,
                                             void *aux_ptr, double *ppart, int tile) {
  using C = cx<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nx = a.nx, F = a.F, cc = a.ccols, S = SC > 0 ? SC : a.S, fst = a.fstride;
  C *buf = reinterpret_cast<C *>(smem_raw);   // [F][fstride >= nx*cc]
  C *twx = buf + (size_t)F * fst;
  double *red = reinterpret_cast<double *>(twx + nx);
  // wave vector k = fx four[0] + fy four[1] + fz four[2] in parts: kxv per x
  // slot, cyv / czv per column of the tile (w = 1 on the axis's Nyquist index)
  V4<T> *kxv = reinterpret_cast<V4<T> *>(red + 64);
  V4<T> *cyv = kxv + nx, *czv = cyv + cc;
  int *csy = reinterpret_cast<int *>(czv + cc), *csz = csy + ((cc + 3) & ~3);
  // Im xi spectrum at this tile's kx = nx/2 points (cc columns x S systems),
  // read once at CTA start: those few points would otherwise make one warp
  // wait on S dependent global loads while the CTA waits for it
  C *nqs = reinterpret_cast<C *>(csz + ((cc + 3) & ~3));
  const size_t col0 = (size_t)tile * cc;
  const size_t ncols = a.ncols;
  const int cpr = (int)(cc * sizeof(C) / 16);    // 16-byte chunks per (field, x) row
  const int nchunks = F * nx * cpr;
  const FastDiv &dc = a.fd_cpr, &dnx = a.fd_nx;
  C *caux = reinterpret_cast<C *>(aux_ptr);
  if (a.mode != PASS_SYNTH) {
    for (int q = threadIdx.x; q < nchunks; q += blockDim.x) {
      const int fx = dc.div(q), ch = q - fx * cpr;
      const int f = dnx.div(fx), x = fx - f * nx;
      const char *src = reinterpret_cast<const char *>(spec + (size_t)fx * ncols + col0) + 16 * ch;
      cp_async16(reinterpret_cast<char *>(buf + (size_t)f * fst + (size_t)x * cc) + 16 * ch, src);
    }
  } else {
    for (int i = threadIdx.x; i < F * fst; i += blockDim.x) buf[i] = mk<C>((T)0, (T)0);
  }
  load_table(twx, a.tw_x, nx);
  {
    const GreenT<T> &g = gt;
    for (int i = threadIdx.x; i < nx + cc; i += blockDim.x) {
      if (i < nx) {
        const int ix = a.kx_of[i];
        const T f = freq_of<T>(ix, nx);
        kxv[i] = V4<T>{f * g.four[0][0], f * g.four[0][1], f * g.four[0][2], (T)(2 * ix == nx ? 1 : 0)};
      } else {
        const int c = i - nx;
        const int col = (int)(col0 + c);
        const int sy = a.fd_nzp.div(col), sz = col - sy * a.nzp;
        const int iy = a.ky_of[sy], iz = a.kz_of[sz];
        const T fy = freq_of<T>(iy, a.ny), fz = freq_of<T>(iz, a.nz);
        cyv[c] = V4<T>{fy * g.four[1][0], fy * g.four[1][1], fy * g.four[1][2], (T)(2 * iy == a.ny ? 1 : 0)};
        czv[c] = V4<T>{fz * g.four[2][0], fz * g.four[2][1], fz * g.four[2][2], (T)(2 * iz == a.nz ? 1 : 0)};
        csy[c] = sy;
        csz[c] = sz;
      }
    }
    if (a.imag == IMAG_NYQ && a.mode != PASS_SYNTH)
      for (int i = threadIdx.x; i < cc * S; i += blockDim.x) {
        const int c = i / S, f = i - c * S;
        const int col = (int)(col0 + c);
        const int sy = a.fd_nzp.div(col), sz = col - sy * a.nzp;
        bool nq;
        const size_t ai = nyq_index<T, C>(a, f, a.sx_n, sy, sz, nq);
        nqs[i] = nq ? caux[ai] : mk<C>((T)0, (T)0);
      }
  }
  // run-time slip count: the contraction's constants staged for vector loads
  constexpr bool STAGED = SC == 0 && PFDD_PENCIL_SMEM_CONST;
  __shared__ __align__(16) T cst_sig[STAGED ? PFDD_MAXS * 6 : 1];
  __shared__ __align__(16) T cst_out[STAGED ? PFDD_MAXS * 12 : 1];
  if constexpr (STAGED) {
    for (int i = threadIdx.x; i < S * 6; i += blockDim.x) {
      const int b = i / 6, q = i - 6 * b;
      cst_sig[i] = gt.sig[b][q];
      cst_out[12 * b + q] = gt.epso[b][q];
      cst_out[12 * b + 6 + q] = gt.sigo[b][q];
    }
  }
  if (a.mode != PASS_SYNTH) cp_async_wait_all();
  __syncthreads();

  Batch gx{F * cc, cc, 1, fst, cc, true, a.fd_fcc, a.fd_cc};
  if (a.mode != PASS_SYNTH) fft_forward<MaxRadix<NT>::value, GeomPencil>(buf, twx, a.px, gx);

  double dsq = 0.0;
  const GreenT<T> &g = gt;
  const size_t fs = (size_t)fst;
  auto gacc = [&](int b, C x, C (&acc)[6]) {
    if constexpr (STAGED) green_accumulate_s<T>(cst_sig, b, x, acc);
    else green_accumulate<T>(g, b, x, acc);
  };
  auto gout = [&](int aa, const C (&sv)[6], const C (&Tq)[6], bool nzk) -> C {
    if constexpr (STAGED) return green_out_s<T>(cst_out, aa, sv, Tq, nzk);
    else return green_out<T>(g, aa, sv, Tq, nzk);
  };
  for (int w = threadIdx.x; w < nx * cc; w += blockDim.x) {
    const int sx = a.fd_cc.div(w), c = w - sx * cc;
    const int sy = csy[c], sz = csz[c];
    C *pk = buf + sx * cc + c;
    if (a.mode == PASS_SYNTH) {
      bool nq;
      for (int f = 0; f < S; ++f) {
        const size_t ai = nyq_index<T, C>(a, f, sx, sy, sz, nq);
        if (nq) pk[(size_t)f * fst] = caux[ai];
      }
      continue;
    }
    if (sz > a.M) continue;   // row padding: nothing to contract
    const V4<T> X = kxv[sx], Y = cyv[c], Z = czv[c];
    const T kx = X.x + (Y.x + Z.x), ky = X.y + (Y.y + Z.y), kz = X.z + (Y.z + Z.z);
    C sr[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) sr[q] = mk<C>((T)0, (T)0);
    {
      // even and odd systems into separate partial sums (shorter dependences)
      C s2[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) s2[q] = mk<C>((T)0, (T)0);
      int b = 0;
#pragma unroll(SC > 0 ? SC / 2 : 1)
      for (; b + 1 < S; b += 2) {
        const C y0 = pk[b * fs], y1 = pk[(b + 1) * fs];
        gacc(b, y0, sr);
        gacc(b + 1, y1, s2);
      }
      if (b < S) gacc(b, pk[b * fs], sr);
#pragma unroll
      for (int q = 0; q < 6; ++q) sr[q] = mk<C>(sr[q].x + s2[q].x, sr[q].y + s2[q].y);
    }
    bool nyq = false;
    size_t a0 = 0, astride = 0;
    if (a.imag == IMAG_NYQ) {
      a0 = nyq_index<T, C>(a, 0, sx, sy, sz, nyq);
      astride = (sz == a.M) ? (size_t)a.nx * a.ny : (sy == a.sy_n ? (size_t)a.nx * a.M : (size_t)a.ny * a.M);
    }
    if (a.imag == IMAG_FULL || nyq || a.imag == IMAG_NONE) {
      // B at the index -k is B evaluated at the wave vector the reference
      // assigns to -k: -f on every axis except at its Nyquist index (frec)
      const T gx = X.w != (T)0 ? (T)1 : (T)-1, gy = Y.w != (T)0 ? (T)1 : (T)-1, gz = Z.w != (T)0 ? (T)1 : (T)-1;
      const T mx = gx * X.x + (gy * Y.x + gz * Z.x), my = gx * X.y + (gy * Y.y + gz * Z.y),
              mz = gx * X.z + (gy * Y.z + gz * Z.z);
      if (a.imag == IMAG_NONE) {
        // real field only: average B over k and index -k (the Hermitian part)
        C Tp[6], Tm[6];
        const bool zp = green_tensor<T>(g, sr, kx, ky, kz, Tp);
        const bool zq = green_tensor<T>(g, sr, mx, my, mz, Tm);
#pragma unroll(SC > 0 ? SC : 1)
        for (int aa = 0; aa < S; ++aa) {
          const C P = gout(aa, sr, Tp, zp), Q = gout(aa, sr, Tm, zq);
          pk[aa * fs] = mk<C>((T)0.5 * (P.x + Q.x), (T)0.5 * (P.y + Q.y));
        }
        continue;
      }
      // P = B(k)(Xr + i Xi), Q = B(k')(Xr - i Xi), k' = vector of index -k;
      // Er = (P + Q)/2, Ei = (P - Q)/(2i): the real and imaginary fields of
      // IFFT(B_index X) for the complex field X = Xr + i Xi.
      // Im xi of the point for system b: the second field (full carrier), the
      // tile's kx = nx/2 snapshot, or the Nyquist spectrum (loads batched by 4)
      const bool snap = a.imag == IMAG_NYQ && sx == a.sx_n;
      const int s0 = c * S;
      C si[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) si[q] = mk<C>((T)0, (T)0);
      for (int b0 = 0; b0 < S; b0 += 4) {
        C xv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int b = b0 + q;
          xv[q] = mk<C>((T)0, (T)0);
          if (b < S) {
            if (a.imag == IMAG_FULL) xv[q] = pk[(S + b) * fs];
            else if (snap) xv[q] = nqs[s0 + b];
            else xv[q] = caux[a0 + b * astride];
          }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (b0 + q < S) gacc(b0 + q, xv[q], si);
      }
      C sp[6], sq[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        sp[q] = mk<C>(sr[q].x - si[q].y, sr[q].y + si[q].x);  // Sr + i Si
        sq[q] = mk<C>(sr[q].x + si[q].y, sr[q].y - si[q].x);  // Sr - i Si
      }
      C Tp[6], Tm[6];
      const bool zp = green_tensor<T>(g, sp, kx, ky, kz, Tp);
      const bool zq = green_tensor<T>(g, sq, mx, my, mz, Tm);
      const T cd = (T)a.cd;
      const double wgt = (sz == 0 || sz == a.M) ? 1.0 : 2.0;   // k and its unstored partner -k
#pragma unroll 1
      for (int aa = 0; aa < S; ++aa) {
        const C P = gout(aa, sp, Tp, zp);
        const C Q = gout(aa, sq, Tm, zq);
        pk[aa * fs] = mk<C>((T)0.5 * (P.x + Q.x), (T)0.5 * (P.y + Q.y));
        // (P - Q)/(2i) = -i (P - Q)/2
        const C ei = mk<C>((T)0.5 * (P.y - Q.y), (T)-0.5 * (P.x - Q.x));
        if (a.imag == IMAG_FULL) {
          pk[(S + aa) * fs] = ei;
        } else if (a.mode == PASS_ENERGY) {
          // 1/2 <Im xi, (L xi)_i> from the Nyquist spectrum (Parseval; 1/N on the host)
          const C xim = caux[a0 + aa * astride];
          dsq += 0.5 * wgt * ((double)xim.x * (double)ei.x + (double)xim.y * (double)ei.y);
        } else {
          // Nyquist point: Im xi spectrum updated in k-space (no mask, no core force on Im xi)
          const C dlt = mk<C>(-cd * ei.x, -cd * ei.y);
          C *ap = caux + a0 + aa * astride;
          C old;
          if (snap) old = nqs[s0 + aa];
          else old = *ap;
          *ap = mk<C>(old.x + dlt.x, old.y + dlt.y);
          dsq += wgt * ((double)dlt.x * (double)dlt.x + (double)dlt.y * (double)dlt.y);
        }
      }
      continue;
    }
    // B(k) = B(index -k) off the Nyquist planes: Er = B Xr
    C Tp[6];
    const bool zp = green_tensor<T>(g, sr, kx, ky, kz, Tp);
    if (SC == 0 && !STAGED && g.tf) {   // (with S unrolled the two-term form's constants are immediates)
      C Z[6];
      green_z<T>(g, sr, Tp, zp, Z);
      int aa = 0;
#pragma unroll(SC > 0 ? SC / 2 : 1)
      for (; aa + 1 < S; aa += 2) {   // two outputs in flight
        const C o0 = green_out_z<T>(g, aa, Z), o1 = green_out_z<T>(g, aa + 1, Z);
        pk[aa * fs] = o0;
        pk[(aa + 1) * fs] = o1;
      }
      if (aa < S) pk[aa * fs] = green_out_z<T>(g, aa, Z);
      continue;
    }
    {
      int aa = 0;
#pragma unroll(SC > 0 ? SC / 2 : 1)
      for (; aa + 1 < S; aa += 2) {   // two outputs in flight
        const C o0 = gout(aa, sr, Tp, zp), o1 = gout(aa + 1, sr, Tp, zp);
        pk[aa * fs] = o0;
        pk[(aa + 1) * fs] = o1;
      }
      if (aa < S) pk[aa * fs] = gout(aa, sr, Tp, zp);
    }
  }
  if (ppart) block_sum2(dsq, 0.0, red, ppart + 2 * tile);
  __syncthreads();

  fft_inverse<MaxRadix<NT>::value, GeomPencil>(buf, twx, a.px, gx);

  for (int q = threadIdx.x; q < nchunks; q += blockDim.x) {
    const int fx = dc.div(q), ch = q - fx * cpr;
    const int f = dnx.div(fx), x = fx - f * nx;
    float4 *dst = reinterpret_cast<float4 *>(reinterpret_cast<char *>(spec + (size_t)fx * ncols + col0) + 16 * ch);
    *dst = *reinterpret_cast<const float4 *>(reinterpret_cast<const char *>(buf + (size_t)f * fst + (size_t)x * cc) +
                                             16 * ch);
  }
}

// grid.x = ncols / ccols tiles; SC: constant slip-system count (0: a.S)
template <typename T, int NT, int SC = 0>
__global__ void __launch_bounds__(NT, (PencilMinBlocks<T>::value)) k_xpencil(cx<T> *__restrict__ spec, PencilArgs a,
                                                const int *__restrict__ stop) {
  if (stop && *stop) return;
  xpencil_body<T, NT, SC>(spec, a, green_t<T>(a.g), a.aux, a.partials, blockIdx.x);
}

// grid = (tiles, instances of the group)
template <typename T, int NT, int SC = 0>
__global__ void __launch_bounds__(NT, (PencilMinBlocks<T>::value)) k_xpencil_tab(const InstPtrs *__restrict__ tab, PencilArgs a) {
  const InstPtrs &ip = tab[blockIdx.y];
  if (ip.flags[0]) return;
  xpencil_body<T, NT, SC>(static_cast<cx<T> *>(ip.spec), a, green_t<T>(a.g), ip.aux, ip.ppart, blockIdx.x);
}

// Slip-system counts with an unrolled contraction (basal / {111} triples 3,
// BCC pairs 2); others, FCC's 12 among them (fully unrolled it spills),
// run the generic loop.
#ifndef PFDD_UNROLL_S12
#define PFDD_UNROLL_S12 0
#endif
template <typename Fn> __host__ inline void with_pencil_sc(int S, Fn f) {
  switch (S) {
    case 3: f(std::integral_constant<int, 3>()); break;
    case 2: f(std::integral_constant<int, 2>()); break;
#if PFDD_UNROLL_S12
    case 12: f(std::integral_constant<int, 12>()); break;
#endif
    default: f(std::integral_constant<int, 0>()); break;
  }
}

// ------------------------------------------------------------ core force
// dE_core for field a at site r from Re xi (App::core_energy dispatch,
// app.cpp:663-672).  k[] holds constants already divided by mu*dslip*b
// (or mu) on the host, in the reference's order of operations.
// Core model 5's coefficient cof(theta) at site r of system a
// (core_energy_bcc_perfect, fft_fftw_slab.cpp:1108-1117), theta from
// FFTW_Slab::gradient (:869-1065): periodic central differences of Re xi_a,
// taken to the global frame through `four` in place (the y and z rows use the
// already transformed x and y components, as the reference does), the line
// direction t = grad x n normalised, theta = acos(t . b), pi - theta when
// (b x t) . n < 0, and theta = -1 (cof = 1) where |t| <= 0.1.
template <typename T>
__device__ __forceinline__ T bcc_cof(const Core &cm, int a, size_t r, size_t N, const T *__restrict__ xin) {
  const int nx = cm.nx, ny = cm.ny, nz = cm.nz;
  const int k = (int)(r % nz), j = (int)((r / nz) % ny), i = (int)(r / ((size_t)nz * ny));
  const T *f = xin + (size_t)a * N;
  auto at = [&](int ii, int jj, int kk) { return f[((size_t)ii * ny + jj) * nz + kk]; };
  const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;
  const int jp = j + 1 == ny ? 0 : j + 1, jm = j == 0 ? ny - 1 : j - 1;
  const int kp = k + 1 == nz ? 0 : k + 1, km = k == 0 ? nz - 1 : k - 1;
  T gx = (at(ip, j, k) - at(im, j, k)) / (T)2;
  T gy = (at(i, jp, k) - at(i, jm, k)) / (T)2;
  T gz = (at(i, j, kp) - at(i, j, km)) / (T)2;
  const double(*F)[3] = cm.four;
  gx = gx * (T)F[0][0] + gy * (T)F[1][0] + gz * (T)F[2][0];
  gy = gx * (T)F[0][1] + gy * (T)F[1][1] + gz * (T)F[2][1];
  gz = gx * (T)F[0][2] + gy * (T)F[1][2] + gz * (T)F[2][2];
  const T n0 = (T)cm.xn[a][0], n1 = (T)cm.xn[a][1], n2 = (T)cm.xn[a][2];
  const T b0 = (T)cm.xb[a][0], b1 = (T)cm.xb[a][1], b2 = (T)cm.xb[a][2];
  T t0 = gy * n2 - gz * n1, t1 = gz * n0 - gx * n2, t2 = gx * n1 - gy * n0;
  const T mag = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
  if (mag <= (T)0.1) return (T)1;
  t0 /= mag;
  t1 /= mag;
  t2 /= mag;
  T th = acos(t0 * b0 + t1 * b1 + t2 * b2);
  const T dir = (b1 * t2 - b2 * t1) * n0 + (b2 * t0 - b0 * t2) * n1 + (b0 * t1 - b1 * t0) * n2;
  if (dir < (T)0) th = acos((T)-1) - th;
  return th < (T)1.23 ? (T)1.1603 * th * th - (T)2.0431 * th + (T)1
                      : (T)0.5473 * th * th - (T)2.0035 * th + (T)1.8923;
}

template <typename T>
__device__ __forceinline__ T core_derivative(const Core &cm, T x, int a, size_t r, size_t N, const T *__restrict__ xin,
                                             const T *__restrict__ site) {
  switch (cm.flag) {
    case 5:   // BCC perfect: usf' cof(theta) pi sin(2 pi x) (fft_fftw_slab.cpp:1120)
      return core_k<T>(cm, 0) * bcc_cof<T>(cm, a, r, N, xin) * sinpi_t<T>((T)2 * x);
    case 1:   // perfect: An' pi sin(2 pi x)
      return core_k<T>(cm, 0) * sinpi_t<T>((T)2 * x);
    case 6:   // USFE(angle,tau): site[0] = An' pi of the current stress state
      return site[0] * sinpi_t<T>((T)2 * x);
    case 3: { // sine: isf' pi sin(2 pi x) + Cn' 2 pi sin(4 pi x)
      T s, c;
      sincospi_t<T>((T)2 * x, &s, &c);
      return core_k<T>(cm, 0) * s + core_k<T>(cm, 1) * ((T)2 * s * c);
    }
    case 103: { // sine with per-site multiplier m: isf' = isf m/s, Cn' = (usf m - isf'/2)/s
      const T m = site[(size_t)a * N + r];
      T s, c;
      sincospi_t<T>((T)2 * x, &s, &c);
      const T isf = core_k<T>(cm, 2) * m;               // isf / s * m
      const T cn = core_k<T>(cm, 3) * m - isf * core_k<T>(cm, 4);  // usf m / s - isf'/(2 s)
      return (T)PFDD_PI_T * isf * s + (T)(2.0 * PFDD_PI_T) * cn * ((T)2 * s * c);
    }
    case 7: { // mpea: A(r)/(mu dslip b) pi sin(2 pi x)
      const T A = site[(size_t)a * N + r];
      return A * core_k<T>(cm, 0) * sinpi_t<T>((T)2 * x);
    }
    case 4: { // pyrII: the reference writes dE_core only at the last site (fft_fftw_slab.cpp:1491)
      if (r != N - 1) return (T)0;
      T acc = (T)0;
#pragma unroll
      for (int n = 1; n <= 4; ++n) {
        T s, c;
        sincospi_t<T>((T)(2 * n) * x, &s, &c);
        acc += (T)(2.0 * n * PFDD_PI_T) * (core_k<T>(cm, 4 + n) * c - core_k<T>(cm, n) * s);
      }
      return acc;
    }
    case 2: { // extended, three systems per plane (fft_fftw_slab.cpp:1300-1352)
      const int p = a / 3, w = a - 3 * p;
      const T x1 = xin[(size_t)(3 * p) * N + r], x2 = xin[(size_t)(3 * p + 1) * N + r],
              x3 = xin[(size_t)(3 * p + 2) * N + r];
      const T c1 = core_k<T>(cm, 0), c2 = core_k<T>(cm, 1), c3 = core_k<T>(cm, 2), c4 = core_k<T>(cm, 3), a1 = core_k<T>(cm, 4),
              a3 = core_k<T>(cm, 5), pre = core_k<T>(cm, 6);
      auto S2 = [](T t) { return sinpi_t<T>((T)2 * t); };
      auto S4 = [](T t) { return sinpi_t<T>((T)4 * t); };
      auto C2 = [](T t) { return cospi_t<T>((T)2 * t); };
      auto C4 = [](T t) { return cospi_t<T>((T)4 * t); };
      const T two = (T)2, three = (T)3;
      T d;
      if (w == 0) {  // df1core
        d = c1 * (S2(x2 - x1) + S2(x3 - x1)) +
            c2 * (two * S2(x2 + x3 - two * x1) + S2(two * x2 - x3 - x1) + S2(two * x3 - x1 - x2)) +
            (two * c3) * (S4(x2 - x1) + S4(x3 - x1)) +
            c4 * (three * S2(x2 + two * x3 - three * x1) + three * S2(two * x2 + x3 - three * x1) +
                  two * S2(three * x2 - x3 - two * x1) + S2(three * x2 - two * x3 - x1) +
                  S2(three * x3 - x1 - two * x2) + two * S2(three * x3 - two * x1 - x2)) +
            a1 * (C2(x1 - x2) - C2(x3 - x1)) + (two * a3) * (C4(x1 - x2) - C4(x3 - x1));
      } else if (w == 1) {  // df2core
        d = c1 * (S2(x1 - x2) + S2(x3 - x2)) +
            c2 * (S2(two * x1 - x2 - x3) + two * S2(x3 + x1 - two * x2) + S2(two * x3 - x1 - x2)) +
            (two * c3) * (S4(x1 - x2) + S4(x3 - x2)) +
            c4 * (S2(three * x1 - x2 - two * x3) + two * S2(three * x1 - two * x2 - x3) +
                  three * S2(x3 + two * x1 - three * x2) + three * S2(two * x3 + x1 - three * x2) +
                  two * S2(three * x3 - x1 - two * x2) + S2(three * x3 - two * x1 - x2)) +
            a1 * (C2(x2 - x3) - C2(x1 - x2)) + (two * a3) * (C4(x2 - x3) - C4(x1 - x2));
      } else {  // df3core
        d = c1 * (S2(x2 - x3) + S2(x1 - x3)) +
            c2 * (S2(two * x1 - x2 - x3) + S2(two * x2 - x3 - x1) + two * S2(x1 + x2 - two * x3)) +
            (two * c3) * (S4(x2 - x3) + S4(x1 - x3)) +
            c4 * (two * S2(three * x1 - x2 - two * x3) + S2(three * x1 - two * x2 - x3) +
                  S2(three * x2 - x3 - two * x1) + two * S2(three * x2 - two * x3 - x1) +
                  three * S2(x1 + two * x2 - three * x3) + three * S2(two * x1 + x2 - three * x3)) +
            a1 * (C2(x3 - x1) - C2(x2 - x3)) + (two * a3) * (C4(x3 - x1) - C4(x2 - x3));
      }
      return pre * d;
    }
    default:
      return (T)0;
  }
}

// ------------------------------------------------------------ core energy
// f(x) per site-slip whose derivative core_derivative evaluates (the reference
// accumulates E_core but never reduces it, fft_fftw_slab.cpp:1399).
template <typename T>
__device__ __forceinline__ T core_energy_density(const Core &cm, T x, int a, size_t r, size_t N,
                                                 const T *__restrict__ site, const T *__restrict__ xin) {
  const T s1 = sinpi_t<T>(x), s2 = sinpi_t<T>((T)2 * x);
  switch (cm.flag) {
    case 5:   // BCC perfect: usf' cof(theta) sin^2(pi x) (fft_fftw_slab.cpp:1119)
      return core_k<T>(cm, 10) * bcc_cof<T>(cm, a, r, N, xin) * s1 * s1;
    case 2: { // extended: fcore of the plane of systems 3p..3p+2 (fft_fftw_slab.cpp:1320), on its first system
      const int p = a / 3;
      if (a != 3 * p) return (T)0;
      const T x1 = xin[(size_t)(3 * p) * N + r], x2 = xin[(size_t)(3 * p + 1) * N + r],
              x3 = xin[(size_t)(3 * p + 2) * N + r];
      auto C2 = [](T t) { return cospi_t<T>((T)2 * t); };
      auto C4 = [](T t) { return cospi_t<T>((T)4 * t); };
      auto S2 = [](T t) { return sinpi_t<T>((T)2 * t); };
      auto S4 = [](T t) { return sinpi_t<T>((T)4 * t); };
      const T two = (T)2, three = (T)3;
      const T e = core_k<T>(cm, 7) +
                  core_k<T>(cm, 0) * (C2(x1 - x2) + C2(x2 - x3) + C2(x3 - x1)) +
                  core_k<T>(cm, 1) * (C2(two * x1 - x2 - x3) + C2(two * x2 - x3 - x1) + C2(two * x3 - x1 - x2)) +
                  core_k<T>(cm, 2) * (C4(x1 - x2) + C4(x2 - x3) + C4(x3 - x1)) +
                  core_k<T>(cm, 3) * (C2(three * x1 - x2 - two * x3) + C2(three * x1 - two * x2 - x3) +
                                      C2(three * x2 - x3 - two * x1) + C2(three * x2 - two * x3 - x1) +
                                      C2(three * x3 - x1 - two * x2) + C2(three * x3 - two * x1 - x2)) +
                  core_k<T>(cm, 4) * (S2(x1 - x2) + S2(x2 - x3) + S2(x3 - x1)) +
                  core_k<T>(cm, 5) * (S4(x1 - x2) + S4(x2 - x3) + S4(x3 - x1));
      return core_k<T>(cm, 8) * e;
    }
    case 1:
      return core_k<T>(cm, 10) * s1 * s1;
    case 6:
      return site[1] * s1 * s1;
    case 3:
      return core_k<T>(cm, 10) * s1 * s1 + core_k<T>(cm, 11) * s2 * s2;
    case 7:
      return site[(size_t)a * N + r] * core_k<T>(cm, 10) * s1 * s1;
    case 103: {
      const T m = site[(size_t)a * N + r];
      const T isf = core_k<T>(cm, 2) * m;
      const T cn = core_k<T>(cm, 3) * m - isf * core_k<T>(cm, 4);
      return isf * s1 * s1 + cn * s2 * s2;
    }
    default:
      return (T)0;
  }
}

// ------------------------------------------------------------ adjoint helpers
// f''(x) and the derivatives of f'(x) with respect to the model's parameters
// p0, p1 (sine: isf, usf; perfect / USFE: An, -; sine field: isf, usf;
// MPEA: none), in J/m^2, with the reference's constants (core_derivative).
template <typename T>
__device__ __forceinline__ void core_adjoint_terms(const Core &cm, T x, int a, size_t r, size_t N,
                                                   const T *__restrict__ site, T &d2, T &dp0, T &dp1) {
  const T pi = (T)PFDD_PI_T;
  T s2, c2, s4, c4;
  sincospi_t<T>((T)2 * x, &s2, &c2);
  s4 = (T)2 * s2 * c2;
  c4 = (T)1 - (T)2 * s2 * s2;
  dp0 = (T)0;
  dp1 = (T)0;
  switch (cm.flag) {
    case 1:
    case 6: {  // k0 = An' pi (site[0] for model 6); f' = k0 sin(2 pi x); d/dAn = (pi/s) sin(2 pi x)
      const T k0 = cm.flag == 6 ? site[0] : core_k<T>(cm, 0);
      d2 = k0 * (T)2 * pi * c2;
      dp0 = core_k<T>(cm, 7) * s2;
      return;
    }
    case 3:  // k0 = isf' pi, k1 = Cn' 2 pi
      d2 = core_k<T>(cm, 0) * (T)2 * pi * c2 + core_k<T>(cm, 1) * (T)4 * pi * c4;
      dp0 = core_k<T>(cm, 7) * s2 - core_k<T>(cm, 8) * s4;   // (pi/s) sin2 - (pi/s^2) sin4
      dp1 = core_k<T>(cm, 9) * s4;                             // (2 pi/s) sin4
      return;
    case 103: {
      const T m = site[(size_t)a * N + r];
      const T isf = core_k<T>(cm, 2) * m;
      const T cn = core_k<T>(cm, 3) * m - isf * core_k<T>(cm, 4);
      d2 = (T)2 * pi * pi * isf * c2 + (T)8 * pi * pi * cn * c4;
      dp0 = m * (core_k<T>(cm, 7) * s2 - core_k<T>(cm, 8) * s4);
      dp1 = m * core_k<T>(cm, 9) * s4;
      return;
    }
    case 7: {
      const T A = site[(size_t)a * N + r];
      d2 = A * core_k<T>(cm, 0) * (T)2 * pi * c2;
      return;
    }
    default:
      d2 = (T)0;
      return;
  }
}

// ------------------------------------------------------------ P3
template <typename T> struct Vec;
template <> struct Vec<float> { using type = float4; static constexpr int n = 4; };
template <> struct Vec<double> { using type = double2; static constexpr int n = 2; };

template <typename T>
__device__ __forceinline__ T update_one(const UpdateArgs &u, bool real_field, int sys, T el, T old, T tau, size_t r,
                                        size_t N, const T *__restrict__ xin, const T *__restrict__ site) {
  const T cd = (T)u.cd;
  if (real_field) {
    const T dE = core_derivative<T>(u.core, old, sys, r, N, xin, site);
    return old - cd * (el - tau + dE);
  }
  return old - cd * el;
}

// ------------------------------------------------------------ register-resident z passes
// The z side of the fused plane pass for a two-stage z plan M = R1 * R2
// (stage A: radix R1 over the whole row, elements j + R2 r; stage B: radix
// R2 over contiguous blocks of R2 slots).  Three passes over shared memory
// replace seven (complex-to-real pairs, two inverse stages, the update's
// read and write, two forward stages, real-to-complex pairs):
//   A  per (row, mirrored block pair): complex-to-real pairs, inverse stage B
//   B  per (row, j): inverse stage A, the per-site update of the 2 R1 real
//      sites the thread then holds (z = 2 (j + R2 r) and + 1), forward stage A
//   C  per (row, mirrored block pair): forward stage B, real-to-complex pairs
// Frequency k = k0 + R1 k1 sits at slot k0 R2 + k1, so the partner M - k of
// block k0 lies in block R1 - k0 (element R2 - 1 - k1), and blocks 0 and
// R1/2 pair with themselves: one work unit holds both blocks of a pair.
template <int M> struct ZPlan {   // the host's make_zplan for the lengths this path compiles
  static constexpr int R1 = (M == 16 || M == 32 || M == 64) ? 8 : (M % 16 == 0) ? 16 : (M % 8 == 0) ? 8 : 4;
  static constexpr int R2 = M / R1;
};
// Calls f(integral_constant<M>) for the z lengths with a register-resident
// path whose host plan is [R1, R2]; returns false otherwise (generic path).
template <typename Fn> __device__ __forceinline__ bool with_zfused(const FftPlan &pz, Fn &&f) {
  auto run = [&](auto Mc) -> bool {
    constexpr int M = decltype(Mc)::value, R1 = ZPlan<M>::R1, R2 = ZPlan<M>::R2;
    if (pz.radix[0] != R1 || pz.nst != (R2 > 1 ? 2 : 1) || (R2 > 1 && pz.radix[1] != R2)) return false;
    f(Mc);
    return true;
  };
  switch (pz.n) {
    case 64: return run(std::integral_constant<int, 64>());
    case 32: return run(std::integral_constant<int, 32>());
    case 16: return run(std::integral_constant<int, 16>());
    case 48: return run(std::integral_constant<int, 48>());
    case 24: return run(std::integral_constant<int, 24>());
    default: return false;
  }
}

// Core models whose force is m (A sin 2 pi x + B sin 4 pi x), A and B
// constant and m = 1 or the per-site field (1 perfect, 3 sine, 6 USFE, 7 MPEA,
// 103 sine with a per-site multiplier): the register-resident z passes inline
// these; the others keep the generic passes.  Adjoint terms in the same form:
// f'' = m (P cos 2 pi x + Q cos 4 pi x), df'/dp0 = m (R sin 2 pi x - S sin 4 pi x),
// df'/dp1 = m U sin 4 pi x (core_adjoint_terms).
__device__ __forceinline__ bool core_sine_family(int flag) {
  return flag == 1 || flag == 3 || flag == 6 || flag == 7 || flag == 103;
}
template <typename T> struct SineCore {
  T A, B, P, Q, R, S, U;
  bool per_site;
};
template <typename T> __device__ __forceinline__ SineCore<T> sine_core(const Core &cm, const T *__restrict__ site) {
  const T pi = (T)PFDD_PI_T;
  SineCore<T> c{(T)0, (T)0, (T)0, (T)0, (T)0, (T)0, (T)0, false};
  const T k0 = core_k<T>(cm, 0), k1 = core_k<T>(cm, 1), k7 = core_k<T>(cm, 7);
  switch (cm.flag) {
    case 1: c.A = k0; c.P = k0 * (T)2 * pi; c.R = k7; break;
    case 6: c.A = site[0]; c.P = site[0] * (T)2 * pi; c.R = k7; break;
    case 3:
      c.A = k0; c.B = k1; c.P = k0 * (T)2 * pi; c.Q = k1 * (T)4 * pi;
      c.R = k7; c.S = core_k<T>(cm, 8); c.U = core_k<T>(cm, 9);
      break;
    case 7: c.per_site = true; c.A = k0; c.P = k0 * (T)2 * pi; break;
    case 103: {
      const T k2 = core_k<T>(cm, 2), cn = core_k<T>(cm, 3) - k2 * core_k<T>(cm, 4);
      c.per_site = true;
      c.A = pi * k2; c.B = (T)2 * pi * cn; c.P = (T)2 * pi * pi * k2; c.Q = (T)8 * pi * pi * cn;
      c.R = k7; c.S = core_k<T>(cm, 8); c.U = core_k<T>(cm, 9);
      break;
    }
    default: break;
  }
  return c;
}

// Thread orders of the z passes.  FP32 rows are 4 words apart in the 32 banks
// (row stride 2 mod 16 complex), so rows y and y + d start 4 d words apart.
// Pass B item w -> (row y, j): in blocks of 8 rows, each half-warp takes
// 16 / R2 rows spaced R2 / 2 apart, whose 2 R2-word runs then tile the banks.
template <int R2> __device__ __forceinline__ void zb_item(int w, int rows, int &y, int &j) {
  if constexpr (R2 == 2 || R2 == 4 || R2 == 8) {
    if ((rows & 7) == 0) {
      constexpr int h = 16 / R2, sp = R2 / 2;
      const int b8 = w / (8 * R2), t = w - b8 * (8 * R2);
      const int rr = t / R2;
      j = t - rr * R2;
      y = 8 * b8 + (rr % h) * sp + rr / h;
      return;
    }
  }
  y = w / R2;
  j = w - y * R2;
}
// Pass A / C unit w -> (row y, unit u), U = R1/2 units per row, each loading
// two blocks of R2 slots as 16-byte chunks: each quarter-warp takes R2 / 2
// consecutive rows x 16 / R2 consecutive units, whose first chunks
// (4 y + 2 R2 u words) then cover the 32 banks once.
template <int R2, int U> __device__ __forceinline__ void zac_item(int w, int rows, int &y, int &u) {
  if constexpr ((R2 == 4 || R2 == 8) && U % (16 / R2) == 0) {
    constexpr int Y = R2 / 2, V = 16 / R2;
    if (rows % Y == 0) {
      const int blk = w / (Y * U), t = w - blk * (Y * U);
      const int inner = t & 7, qi = t >> 3;
      y = blk * Y + inner % Y;
      u = qi * V + inner / Y;
      return;
    }
  }
  y = w / U;
  u = w - y * U;
}

template <int R2, typename C> __device__ __forceinline__ void zload_block(const C *p, C (&v)[R2]) {
  if constexpr (sizeof(C) == 8 && R2 % 2 == 0) {
#pragma unroll
    for (int r = 0; r < R2; r += 2) {
      const float4 q = reinterpret_cast<const float4 *>(p)[r / 2];
      v[r] = mk<C>(q.x, q.y);
      v[r + 1] = mk<C>(q.z, q.w);
    }
  } else {
#pragma unroll
    for (int r = 0; r < R2; ++r) v[r] = p[r];
  }
}
template <int R2, typename C> __device__ __forceinline__ void zstore_block(C *p, const C (&v)[R2]) {
  if constexpr (sizeof(C) == 8 && R2 % 2 == 0) {
#pragma unroll
    for (int r = 0; r < R2; r += 2)
      reinterpret_cast<float4 *>(p)[r / 2] = make_float4(v[r].x, v[r].y, v[r + 1].x, v[r + 1].y);
  } else {
#pragma unroll
    for (int r = 0; r < R2; ++r) p[r] = v[r];
  }
}

// complex-to-real pair (k, M-k) before the inverse z transform:
// A = X[k] + conj X[M-k], D = X[k] - conj X[M-k], Zin[k] = A + i D conj(W^k),
// Zin[M-k] = conj(A - i D conj(W^k)) (same formulas as the generic loop)
template <typename C> __device__ __forceinline__ void c2r_pair(C &xk, C &xm, const C w, bool self) {
  const C A = mk<C>(xk.x + xm.x, xk.y - xm.y);
  const C D = mk<C>(xk.x - xm.x, xk.y + xm.y);
  const C wd = cmulc(D, w);
  const C iwd = mk<C>(-wd.y, wd.x);
  const C nk = cadd(A, iwd);
  if (!self) xm = cconj(csub(A, iwd));
  xk = nk;
}
// real-to-complex pair (k, M-k) after the forward z transform:
// E = (Zk + conj Zm)/2, O = (Zk - conj Zm)/(2i), X[k] = E + W^k O, X[M-k] = conj(E - W^k O)
template <typename C> __device__ __forceinline__ void r2c_pair(C &zk, C &zm, const C w, bool self) {
  using T = decltype(C::x);
  const C e = mk<C>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y));
  const C o = mk<C>((T)0.5 * (zk.y + zm.y), (T)-0.5 * (zk.x - zm.x));
  const C wo = cmul(w, o);
  const C nk = cadd(e, wo);
  if (!self) zm = cconj(csub(e, wo));
  zk = nk;
}

// Pass A (INV) or C (!INV) over the rows of this CTA; ends with no barrier.
template <bool INV, int M, typename C>
__device__ __forceinline__ void zpass_pairs(C *buf, const C *__restrict__ twr, int rows, int nzs) {
  constexpr int R1 = ZPlan<M>::R1, R2 = ZPlan<M>::R2, U = R1 / 2;
  for (int w = threadIdx.x; w < rows * U; w += blockDim.x) {
    int y, u;
    zac_item<R2, U>(w, rows, y, u);
    C *row = buf + (size_t)y * nzs;
    const int ba = u, bb = u == 0 ? R1 / 2 : R1 - u;
    C a[R2], b[R2];
    zload_block<R2>(row + ba * R2, a);
    zload_block<R2>(row + bb * R2, b);
    if constexpr (!INV) {
      dft<R2, -1>(a);
      dft<R2, -1>(b);
    }
    auto pair = [&](C &p, C &q, int k, bool self) {
      if constexpr (INV) c2r_pair(p, q, twr[k], self);
      else r2c_pair(p, q, twr[k], self);
    };
    if (u == 0) {
      // block 0 (k = R1 k1): k1 = 0 holds x0 + i xM (DC and Nyquist), k1 pairs with R2 - k1
      a[0] = mk<C>(a[0].x + a[0].y, a[0].x - a[0].y);
#pragma unroll
      for (int k1 = 1; 2 * k1 <= R2; ++k1) pair(a[k1], a[R2 - k1], R1 * k1, 2 * k1 == R2);
      // block R1/2 (k = R1/2 + R1 k1): k1 pairs with R2 - 1 - k1
#pragma unroll
      for (int k1 = 0; 2 * k1 <= R2 - 1; ++k1) pair(b[k1], b[R2 - 1 - k1], R1 / 2 + R1 * k1, 2 * k1 == R2 - 1);
    } else {
#pragma unroll
      for (int k1 = 0; k1 < R2; ++k1) pair(a[k1], b[R2 - 1 - k1], u + R1 * k1, false);
    }
    if constexpr (INV) {
      dft<R2, 1>(a);
      dft<R2, 1>(b);
    }
    zstore_block<R2>(row + ba * R2, a);
    zstore_block<R2>(row + bb * R2, b);
  }
}

// Per-instance pointers travel as arguments so the constant parameter block
// (PlaneArgs, UpdateArgs) is read in place and never copied.
// FUSE 1 (PASS_STEP) / 2 (PASS_ADJOINT): only that pass is compiled, and the
// updated plane also stays in shared memory and,
// when `fwd`, is transformed forward (fwd_planes_compute) and stored over the
// spectrum rows this CTA read, as the next step's P1 output.
template <typename T, int NT, bool SPLIT, int FUSE = 0>
__device__ __forceinline__ void inv_update_body(const cx<T> *spec, const T *__restrict__ xin,
                                                T *__restrict__ xout, const PlaneArgs &a, const UpdateArgs &u,
                                                double *__restrict__ partials, size_t plane,
                                                const double *__restrict__ tau_p, const uint8_t *__restrict__ mask,
                                                const void *site_p, int *err, bool fwd = false) {
  using C = cx<T>;
  using V = typename Vec<T>::type;
  constexpr int VN = Vec<T>::n;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int ny = a.ny, nz = a.nz, nzp = a.nzp, nzs = a.nzs, M = a.M;
  const int rows = SPLIT ? ny / 2 : ny;
  const int row0 = row0_of_block<SPLIT>(ny);
  const PlaneSmem<C> sm(smem_raw, a, rows);
  const int stall = stall_switch(err);
  if (threadIdx.x == 0) {
    mbar_init(sm.bar, 1 + stall);
    // the update reads this CTA's xi rows after the transforms: start them towards L2 now
    if (u.mode != PASS_SYNTH) prefetch_l2_bulk(xin + (plane * ny + row0) * nz, (uint32_t)(rows * nz * sizeof(T)));
  }
  __syncthreads();
  // spectrum rows of nzp entries -> shared rows of nzs (bulk copies, one warp)
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) mbar_expect_tx(sm.bar, (uint32_t)((size_t)rows * nzp * sizeof(C)));
    __syncwarp();
    const C *src = spec + (plane * (size_t)ny + row0) * nzp;
    if (nzs == nzp) {
      if (threadIdx.x == 0) bulk_g2s(sm.buf, src, (uint32_t)((size_t)rows * nzp * sizeof(C)), sm.bar);
    } else {
      for (int y = threadIdx.x; y < rows; y += 32)
        bulk_g2s(sm.buf + (size_t)y * nzs, src + (size_t)y * nzp, (uint32_t)(nzp * sizeof(C)), sm.bar);
    }
  }
  load_plane_tables(sm, a);
  __syncthreads();
  const bool ok = plane_wait(sm.bar, stall, err);
  // after a timeout a split CTA carries on without storing: its peer waits at the cluster barriers
  if (!ok && !SPLIT) return;
  C *buf = sm.buf;
  const C *twr = sm.twr;
  const int *pos = sm.pos;

  // pack the kz = 0 and kz = nz/2 columns into slot 0: Y0 + i YM
  for (int y = threadIdx.x; y < rows; y += blockDim.x) {
    C *row = buf + (size_t)y * nzs;
    const C y0 = row[0], ym = row[M];
    row[0] = mk<C>(y0.x - ym.y, y0.y + ym.x);
  }
  __syncthreads();
  Batch gy{M, M, 1, 0, nzs, true, a.fd_m, a.fd_m};
  fft_inverse<MaxRadix<NT>::value, GeomCols>(buf, SPLIT ? sm.twy + rows : sm.twy, a.py, gy);
  if constexpr (SPLIT) cross_stage<true>(buf, sm.twy, rows, a.fd_m, nzs);

  const int f = (int)(plane / a.nx);
  const int x = (int)(plane - (size_t)f * a.nx);
  const bool real_field = f < u.S;
  const int sys = real_field ? f : f - u.S;
  const size_t N = (size_t)a.nx * ny * nz;
  const size_t off = (plane * (size_t)ny + row0) * nz;   // first site of this CTA's rows
  const size_t rbase = ((size_t)x * ny + row0) * nz;
  const T invN = (T)u.invN;

  // Update (FUSE 1) and adjoint (FUSE 2) passes of a two-stage z plan: the
  // register-resident z passes A, B, C (see zpass_pairs).
  bool zdone = false;
  if constexpr (FUSE != 0) {
    // (only when pass B, rows x R2 work items, keeps every thread busy in FP64
    // or half of them in FP32: measured on 64^3 FP64 and 128x128x32 FP32)
    const bool done = a.zfused && (FUSE == 1 || u.mode == PASS_ADJOINT) && core_sine_family(u.core.flag) &&
                      (sizeof(T) == 4 ? 2 : 1) * rows * (a.pz.n / a.pz.radix[0]) >= (int)blockDim.x &&
                      with_zfused(a.pz, [&](auto Mc) {
      constexpr int MM = decltype(Mc)::value, R1 = ZPlan<MM>::R1, R2 = ZPlan<MM>::R2;
      zpass_pairs<true, MM>(buf, twr, rows, nzs);
      __syncthreads();
      const C *twz = sm.twz;
      const T *site = reinterpret_cast<const T *>(site_p);
      const SineCore<T> sc = sine_core<T>(u.core, site);
      const T *srow = sc.per_site ? site + (size_t)sys * N + rbase : nullptr;
      const uint8_t *mrow = mask ? mask + (size_t)sys * N + rbase : nullptr;
      const T cdt = (T)u.cd;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};   // FUSE 1: |dxi|^2, sum xi; FUSE 2: the gradient sums
      // B: inverse stage A, the per-site pass on the 2 R1 sites z = 2 (j + R2 r) + {0, 1}, forward stage A
      for (int w = threadIdx.x; w < rows * R2; w += blockDim.x) {
        int y, j;
        zb_item<R2>(w, rows, y, j);
        C *row = buf + (size_t)y * nzs;
        const int base = y * nz + 2 * j;   // site of element j in this CTA's rows
        // the item's old values first: their global loads are in flight during the transform
        C ol[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) ol[r] = *reinterpret_cast<const C *>(xin + off + base + 2 * R2 * r);
        C v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = row[j + R2 * r];
        apply_twiddles<R1, true>(v, twz, j);
        dft<R1, 1>(v);
        T s0 = (T)0, s1 = (T)0, s2 = (T)0;   // four sites' sums in the compute precision, then FP64
#pragma unroll
        for (int r = 0; r < R1; ++r) {
          const int idx = base + 2 * R2 * r;
          const C o = ol[r];
          C m2 = mk<C>((T)1, (T)1);
          if (real_field && srow) m2 = *reinterpret_cast<const C *>(srow + idx);
          const T ov[2] = {o.x, o.y}, ev[2] = {v[r].x * invN, v[r].y * invN}, mv[2] = {m2.x, m2.y};
          T nv[2];
          if constexpr (FUSE == 1) {
            const T tau = real_field ? (T)tau_p[sys] : (T)0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              if (real_field) {
                T sv, cv;
                sincospi_t<T>((T)2 * ov[q], &sv, &cv);
                T force = sc.A * sv + sc.B * ((T)2 * sv * cv);
                if (srow) force *= mv[q];
                nv[q] = ov[q] - cdt * (ev[q] - tau + force);
              } else {
                nv[q] = ov[q] - cdt * ev[q];
              }
              if (mrow && mrow[idx + q]) nv[q] = ov[q];
              const T d = nv[q] - ov[q];
              s0 = fma_t(d, d, s0);
              s1 += nv[q];
            }
          } else {
            // lam_n = lam_{n+1} - cd (L lam + f''(xi_n) lam_{n+1}) on unmasked sites;
            // the parameter gradients use lam_{n+1} and xi_n on the same sites
            C xv2 = mk<C>((T)0, (T)0);
            if (real_field) xv2 = *reinterpret_cast<const C *>(reinterpret_cast<const T *>(u.xfwd) +
                                                                (size_t)sys * N + rbase + idx);
            const T xv[2] = {xv2.x, xv2.y};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const bool frozen = mrow && mrow[idx + q];
              if (real_field) {
                T sa, ca;
                sincospi_t<T>((T)2 * xv[q], &sa, &ca);
                const T s4 = (T)2 * sa * ca, c4 = (T)1 - (T)2 * sa * sa;
                T d2 = sc.P * ca + sc.Q * c4, dp0 = sc.R * sa - sc.S * s4, dp1 = sc.U * s4;
                if (srow) {
                  d2 *= mv[q];
                  dp0 *= mv[q];
                  dp1 *= mv[q];
                }
                nv[q] = frozen ? ov[q] : ov[q] - cdt * (ev[q] + d2 * ov[q]);
                if (!frozen) {
                  s0 = fma_t(ov[q], dp0, s0);
                  s1 = fma_t(ov[q], dp1, s1);
                  s2 += ov[q];
                }
              } else {
                nv[q] = frozen ? ov[q] : ov[q] - cdt * ev[q];
              }
            }
          }
          if (r & 1) {
            acc[0] += (double)s0;
            acc[1] += (double)s1;
            acc[2] += (double)s2;
            s0 = s1 = s2 = (T)0;
          }
          v[r] = mk<C>(nv[0], nv[1]);
          if (ok) *reinterpret_cast<C *>(xout + off + idx) = v[r];
        }
        if (fwd) {
          dft<R1, -1>(v);
          apply_twiddles<R1, false>(v, twz, j);
#pragma unroll
          for (int r = 0; r < R1; ++r) row[j + R2 * r] = v[r];
        }
      }
      if constexpr (FUSE == 1) {
        double vv[2] = {acc[0], real_field ? acc[1] : 0.0};
        plane_sum_slots<SPLIT>(vv, sm.red, partials, plane);
      } else {
        plane_sum<SPLIT, 4, true>(acc, sm.red, u.gpart + 4 * plane);   // summed over the backward steps
      }
      if (fwd) {
        // C: forward stage B and the real-to-complex pairs; zero row padding
        __syncthreads();
        zpass_pairs<false, MM>(buf, twr, rows, nzs);
        for (int y = threadIdx.x; y < rows; y += blockDim.x)
          for (int q = a.nzh; q < a.nzp; ++q) buf[(size_t)y * nzs + q] = mk<C>((T)0, (T)0);
      }
    });
    zdone = done;
  }

  // the generic passes; returns whether the forward y side follows
  auto generic = [&]() -> bool {
  // complex-to-real packing: Zin[k] = A + i w D, Zin[M-k] = conj(A - i w D),
  // A = X[k] + conj X[M-k], D = X[k] - conj X[M-k], w = exp(+2 pi i k / nz)
  // k = 0, one row per thread: slot 0 holds x0 + i xM (the real kz = 0 and
  // kz = nz/2 columns), so Zin[0] = (x0 + xM) + i (x0 - xM)
  for (int y = threadIdx.x; y < rows; y += blockDim.x) {
    C *row = buf + (size_t)y * nzs;
    const C z = row[pos[0]];
    row[pos[0]] = mk<C>(z.x + z.y, z.x - z.y);
  }
  // pairs (k, M-k), k = 1..M/2 taken in slot order (few bank conflicts)
  const int mh = M / 2;
  const int *kord = sm.kord;
  for (int w = threadIdx.x; w < rows * mh; w += blockDim.x) {
    const int y = a.fd_mh.div(w), k = kord[w - y * mh];
    C *row = buf + (size_t)y * nzs;
    const int pk = pos[k];
    const int pm = pos[M - k];
    const C xk = row[pk];
    const C xm = row[pm];
    const C A = mk<C>(xk.x + xm.x, xk.y - xm.y);
    const C D = mk<C>(xk.x - xm.x, xk.y + xm.y);
    const C wd = cmulc(D, twr[k]);            // D * conj(W^k) = D * exp(+2 pi i k/nz)
    const C iwd = mk<C>(-wd.y, wd.x);
    row[pk] = cadd(A, iwd);
    if (pm != pk) row[pm] = cconj(csub(A, iwd));
  }
  __syncthreads();

  Batch gz{rows, rows, nzs, 0, 1, false, a.fd_rows, a.fd_rows};
  fft_inverse<MaxRadix<NT>::value, GeomRows>(buf, sm.twz, a.pz, gz);

  // fused GSFE force + applied stress + masked explicit Euler update,
  // VN consecutive z per thread, two vectors in flight per iteration
  const T *bufr = reinterpret_cast<const T *>(buf);
  const int nvec = nz / VN;
  const int total = rows * nvec;
  const FastDiv &dv = a.fd_nvec;
  if (FUSE == 0 && u.mode == PASS_SYNTH) {
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int y = dv.div(i), zq = i - y * nvec;
      T e[VN];
      *reinterpret_cast<V *>(e) = *reinterpret_cast<const V *>(bufr + (size_t)y * 2 * nzs + zq * VN);
#pragma unroll
      for (int q = 0; q < VN; ++q) e[q] *= invN;
      if (ok) *reinterpret_cast<V *>(xout + off + y * nz + zq * VN) = *reinterpret_cast<V *>(e);
    }
    return false;
  }
  if (FUSE == 0 && u.mode == PASS_ENERGY) {
    // 1/2 xi . (L xi), f(Re xi) and -tau Re xi, summed over the plane (FP64)
    const T *site = reinterpret_cast<const T *>(site_p);
    const double tau = real_field ? tau_p[sys] : 0.0;
    double e_el = 0.0, e_core = 0.0, e_app = 0.0;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int y = dv.div(i), zq = i - y * nvec;
      const int idx = y * nz + zq * VN;
      T xv[VN], e[VN];
      *reinterpret_cast<V *>(xv) = *reinterpret_cast<const V *>(xin + off + idx);
      *reinterpret_cast<V *>(e) = *reinterpret_cast<const V *>(bufr + (size_t)y * 2 * nzs + zq * VN);
#pragma unroll
      for (int q = 0; q < VN; ++q) {
        const double x = (double)xv[q];
        e_el += 0.5 * x * (double)(e[q] * invN);
        if (real_field) {
          e_core += (double)core_energy_density<T>(u.core, xv[q], sys, rbase + idx + q, N, site, xin);
          e_app -= tau * x;
        }
      }
    }
    double v[4] = {e_el, e_core, e_app, 0.0};
    plane_sum<SPLIT>(v, sm.red, u.gpart + 4 * plane);
    return false;
  }
  if (FUSE != 1 && u.mode == PASS_ADJOINT) {
    // lam_n = lam_{n+1} - cd (L lam + f''(xi_n) lam_{n+1}) on unmasked sites
    // (the elastic operator is self-adjoint; tau is constant and drops out);
    // parameter gradients use lam_{n+1} and xi_n on the same sites.
    const T *site = reinterpret_cast<const T *>(site_p);
    const T *xf = reinterpret_cast<const T *>(u.xfwd);
    const T cd = (T)u.cd;
    double g0 = 0.0, g1 = 0.0, gl = 0.0;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int y = dv.div(i), zq = i - y * nvec;
      const int idx = y * nz + zq * VN;
      T lam[VN], e[VN], nv[VN], xv[VN];
      *reinterpret_cast<V *>(lam) = *reinterpret_cast<const V *>(xin + off + idx);
      *reinterpret_cast<V *>(e) = *reinterpret_cast<const V *>(bufr + (size_t)y * 2 * nzs + zq * VN);
      if (real_field) *reinterpret_cast<V *>(xv) = *reinterpret_cast<const V *>(xf + (size_t)sys * N + rbase + idx);
      // the vector's gradient terms summed in the compute precision, then added in FP64
      T v0 = (T)0, v1 = (T)0, vl = (T)0;
#pragma unroll
      for (int q = 0; q < VN; ++q) {
        const size_t r = rbase + idx + q;
        const bool frozen = mask && mask[(size_t)sys * N + r];
        if (real_field) {
          T d2, dp0, dp1;
          core_adjoint_terms<T>(u.core, xv[q], sys, r, N, site, d2, dp0, dp1);
          nv[q] = frozen ? lam[q] : lam[q] - cd * (e[q] * invN + d2 * lam[q]);
          if (!frozen) {
            v0 = fma_t(lam[q], dp0, v0);
            v1 = fma_t(lam[q], dp1, v1);
            vl += lam[q];
          }
        } else {
          nv[q] = frozen ? lam[q] : lam[q] - cd * e[q] * invN;
        }
      }
      g0 += (double)v0;
      g1 += (double)v1;
      gl += (double)vl;
      if (ok) *reinterpret_cast<V *>(xout + off + idx) = *reinterpret_cast<V *>(nv);
      if (FUSE == 2 && fwd)
        *reinterpret_cast<V *>(reinterpret_cast<T *>(buf) + (size_t)y * 2 * nzs + zq * VN) =
            *reinterpret_cast<V *>(nv);
    }
    double v[4] = {g0, g1, gl, 0.0};
    plane_sum<SPLIT, 4, true>(v, sm.red, u.gpart + 4 * plane);   // summed over the backward steps
    if constexpr (FUSE == 2) {
      if (fwd) {   // the next backward step's spectrum of the new lambda
        __syncthreads();
        fwd_planes_z<T, NT>(sm, a, rows);
      }
      return fwd;
    }
    return false;
  }
  if constexpr (FUSE == 2) return false;
  else {
  // update pass only: tau, mask and per-site GSFE are read from here on
  const T tau = real_field ? (T)tau_p[sys] : (T)0;
  const T *site = reinterpret_cast<const T *>(site_p);
  T *bufw = reinterpret_cast<T *>(buf);
  const bool keep = FUSE == 1 && fwd;   // new xi also into shared memory for the forward part
  double dsq = 0.0, sum = 0.0;
  // CF: the core model as a compile-time constant (3: sine GSFE, the common
  // case, with its force inlined), 0: dispatch per site
  auto update_loop = [&](auto CFc) {
  constexpr int CF = decltype(CFc)::value;
  const T cdt = (T)u.cd, k0 = core_k<T>(u.core, 0), k1 = core_k<T>(u.core, 1);
  for (int i0 = threadIdx.x; i0 < total; i0 += 2 * blockDim.x) {
    V oldv[2], elv[2];
    int idx[2], soff[2];
    bool on[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = i0 + h * blockDim.x;
      on[h] = i < total;
      const int y = dv.div(on[h] ? i : 0), zq = (on[h] ? i : 0) - y * nvec;
      idx[h] = y * nz + zq * VN;
      soff[h] = y * 2 * nzs + zq * VN;
      oldv[h] = *reinterpret_cast<const V *>(xin + off + idx[h]);
      elv[h] = *reinterpret_cast<const V *>(bufr + soff[h]);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!on[h]) continue;
      T o[VN], e[VN], nv[VN];
      *reinterpret_cast<V *>(o) = oldv[h];
      *reinterpret_cast<V *>(e) = elv[h];
      // the vector's |dxi|^2 and sum in compute precision, then FP64
      T dq = (T)0, sq = (T)0;
#pragma unroll
      for (int q = 0; q < VN; ++q) {
        const size_t r = rbase + idx[h] + q;
        if constexpr (CF == 3) {
          T sv, cv;
          sincospi_t<T>((T)2 * o[q], &sv, &cv);
          nv[q] = real_field ? o[q] - cdt * (e[q] * invN - tau + (k0 * sv + k1 * ((T)2 * sv * cv)))
                             : o[q] - cdt * (e[q] * invN);
        } else {
          nv[q] = update_one<T>(u, real_field, sys, e[q] * invN, o[q], tau, r, N, xin, site);
        }
        if (mask && mask[(size_t)sys * N + r]) nv[q] = o[q];
        const T d = nv[q] - o[q];
        dq = fma_t(d, d, dq);
        sq += nv[q];
      }
      dsq += (double)dq;
      if (real_field) sum += (double)sq;
      if (ok) *reinterpret_cast<V *>(xout + off + idx[h]) = *reinterpret_cast<V *>(nv);
      if (keep) *reinterpret_cast<V *>(bufw + soff[h]) = *reinterpret_cast<V *>(nv);
    }
  }
  };
  if (u.core.flag == 3) update_loop(std::integral_constant<int, 3>());
  else update_loop(std::integral_constant<int, 0>());
  double v[2] = {dsq, sum};
  plane_sum_slots<SPLIT>(v, sm.red, partials, plane);
  if constexpr (FUSE == 1) {
    if (fwd) {
      __syncthreads();
      fwd_planes_z<T, NT>(sm, a, rows);
    }
    return fwd;
  }
  return false;
  }
  };
  const bool tail = zdone ? fwd : generic();
  // the forward y side of the next step's spectrum (one call site per kernel)
  if constexpr (FUSE != 0) {
    if (tail) fwd_planes_tail<T, NT, SPLIT>(sm, a, const_cast<cx<T> *>(spec), plane, rows, row0, ok);
  }
}

// grid.x = F * nx planes (SPLIT: 2 F nx CTAs in clusters of 2)
template <typename T, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, SPLIT>::value)) k_inv_update(const cx<T> *__restrict__ spec, const T *__restrict__ xin,
                                                   T *__restrict__ xout, PlaneArgs a, UpdateArgs u,
                                                   double *__restrict__ partials) {
  if (u.stop && *u.stop) return;
  inv_update_body<T, NT, SPLIT>(spec, xin, xout, a, u, partials, plane_of_block<SPLIT>(), u.tau, u.mask, u.site,
                                u.err);
}

// P3 of step n fused with P1 of step n + 1 (PASS_STEP): inverse transforms,
// update, then (fwd != 0) the forward transforms of the new plane, stored
// over the same spectrum rows.  grid.x = F * nx planes (x 2 for SPLIT).
template <typename T, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, SPLIT>::value))
    k_step_planes(cx<T> *spec, const T *__restrict__ xin, T *__restrict__ xout, PlaneArgs a, UpdateArgs u,
                  double *__restrict__ partials, int fwd) {
  if (u.stop && *u.stop) return;
  inv_update_body<T, NT, SPLIT, 1>(spec, xin, xout, a, u, partials, plane_of_block<SPLIT>(), u.tau, u.mask,
                                      u.site, u.err, fwd != 0);
}

// One adjoint iteration (PASS_ADJOINT) fused with the forward transforms of
// the new lambda (fwd != 0), for the next backward iteration.
template <typename T, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, SPLIT>::value))
    k_adj_planes(cx<T> *spec, const T *__restrict__ xin, T *__restrict__ xout, PlaneArgs a, UpdateArgs u,
                 double *__restrict__ partials, int fwd) {
  if (u.stop && *u.stop) return;
  inv_update_body<T, NT, SPLIT, 2>(spec, xin, xout, a, u, partials, plane_of_block<SPLIT>(), u.tau, u.mask,
                                   u.site, u.err, fwd != 0);
}

// grid = (F * nx planes [x 2 for SPLIT], instances of the group)
template <typename T, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, SPLIT>::value))
    k_step_planes_tab(const InstPtrs *__restrict__ tab, PlaneArgs a, UpdateArgs u, int fwd) {
  const InstPtrs &ip = tab[blockIdx.y];
  if (ip.flags[0]) return;
  const int cur = ip.flags[4];
  inv_update_body<T, NT, SPLIT, 1>(static_cast<const cx<T> *>(ip.spec), static_cast<const T *>(ip.xi[cur]),
                                      static_cast<T *>(ip.xi[cur ^ 1]), a, u, ip.partials,
                                      plane_of_block<SPLIT>(), ip.tau, ip.mask, ip.site, ip.flags + 3, fwd != 0);
}

// grid = (F * nx planes, instances of the group); per-instance stress, mask,
// GSFE field and buffers come from the table
template <typename T, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, SPLIT>::value)) k_inv_update_tab(const InstPtrs *__restrict__ tab, PlaneArgs a, UpdateArgs u) {
  const InstPtrs &ip = tab[blockIdx.y];
  if (ip.flags[0]) return;
  const int cur = ip.flags[4];
  inv_update_body<T, NT, SPLIT>(static_cast<const cx<T> *>(ip.spec), static_cast<const T *>(ip.xi[cur]),
                                static_cast<T *>(ip.xi[cur ^ 1]), a, u, ip.partials, plane_of_block<SPLIT>(),
                                ip.tau, ip.mask, ip.site, ip.flags + 3);
}

// ------------------------------------------------------------ mixed-size batches
// Groups of one merge class (the same slip systems, material, core model and
// carrier, any grid size) advance in one launch per pass: blockIdx.x maps to
// (group, instance, plane or column tile) through the prefix table
// MultiLaunch::starts (CTAs before each group), and each CTA copies its group's
// geometry (plans, sizes, tables, divisors) into shared memory at its start.
// The planes run whole (no 2-CTA clusters): a batch fills the SMs by count.
constexpr int kMaxMerged = 16;
struct MultiLaunch {
  int ngroups;
  int starts[kMaxMerged + 1];
};
struct MultiPlaneGroup {
  PlaneArgs a;
  UpdateArgs u;
  const InstPtrs *tab;
  int per_member;       // CTAs per instance: F * nx planes
};
struct MultiPencilGroup {
  PencilArgs a;         // only the geometry before `g` is read (one Green table per launch)
  const InstPtrs *tab;
  int per_member;       // column tiles per instance
};
struct MultiFinalGroup {
  const InstPtrs *tab;
  int nparts, nparts2;
  double scale2;
};

__device__ __forceinline__ int group_of_block(const MultiLaunch &m) {
  int g = 0;
  while (g + 1 < m.ngroups && (int)blockIdx.x >= m.starts[g + 1]) ++g;
  return g;
}
// bytes (a multiple of 4) from global to shared memory by the CTA's threads
__device__ __forceinline__ void copy_words(void *dst, const void *src, int bytes) {
  const int *sp = static_cast<const int *>(src);
  int *dp = static_cast<int *>(dst);
  for (int i = threadIdx.x; i < bytes / 4; i += blockDim.x) dp[i] = sp[i];
}

// The fused plane pass of every group of a merge class (P3 of this step and,
// when fwd, P1 of the next).  Static shared memory holds the group's
// arguments; the dynamic part is the plane buffer of the largest group.
template <typename T, int NT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, true>::value))
    k_step_planes_multi(const MultiPlaneGroup *__restrict__ groups, MultiLaunch m, int fwd) {
  __shared__ __align__(16) unsigned char graw[sizeof(MultiPlaneGroup)];
  const MultiPlaneGroup &G = *reinterpret_cast<const MultiPlaneGroup *>(graw);
  const int gi = group_of_block(m);
  copy_words(graw, groups + gi, (int)sizeof(MultiPlaneGroup));
  __syncthreads();
  const int local = (int)blockIdx.x - m.starts[gi];
  const int member = local / G.per_member, plane = local - member * G.per_member;
  const InstPtrs &ip = G.tab[member];
  if (ip.flags[0]) return;
  const int cur = ip.flags[4];
  inv_update_body<T, NT, false, 1>(static_cast<const cx<T> *>(ip.spec), static_cast<const T *>(ip.xi[cur]),
                                   static_cast<T *>(ip.xi[cur ^ 1]), G.a, G.u, ip.partials, (size_t)plane,
                                   ip.tau, ip.mask, ip.site, ip.flags + 3, fwd != 0);
}

// The forward plane pass that opens a run, for every group of a merge class.
template <typename T, int NT>
__global__ void __launch_bounds__(NT, (PlaneMinBlocks<T, true>::value))
    k_fwd_planes_multi(const MultiPlaneGroup *__restrict__ groups, MultiLaunch m) {
  __shared__ __align__(16) unsigned char graw[sizeof(MultiPlaneGroup)];
  const MultiPlaneGroup &G = *reinterpret_cast<const MultiPlaneGroup *>(graw);
  const int gi = group_of_block(m);
  copy_words(graw, groups + gi, (int)sizeof(MultiPlaneGroup));
  __syncthreads();
  const int local = (int)blockIdx.x - m.starts[gi];
  const int member = local / G.per_member, plane = local - member * G.per_member;
  const InstPtrs &ip = G.tab[member];
  if (ip.flags[0]) return;
  fwd_planes_body<T, NT, false>(static_cast<const T *>(ip.xi[ip.flags[4]]), static_cast<cx<T> *>(ip.spec), G.a,
                                ip.flags + 3, (size_t)plane);
}

// The x-pencil pass of every group of a merge class; gt: the contraction's
// constants, equal across the class.
template <typename T, int NT, int SC>
__global__ void __launch_bounds__(NT, (PencilMinBlocks<T>::value))
    k_xpencil_multi(const MultiPencilGroup *__restrict__ groups, MultiLaunch m, const __grid_constant__ GreenT<T> gt) {
  constexpr int kGeom = (int)offsetof(PencilArgs, g);
  __shared__ __align__(16) unsigned char araw[(kGeom + 15) & ~15];
  const PencilArgs &A = *reinterpret_cast<const PencilArgs *>(araw);
  const int gi = group_of_block(m);
  copy_words(araw, &groups[gi].a, kGeom & ~3);
  __syncthreads();
  const int local = (int)blockIdx.x - m.starts[gi];
  const int per = groups[gi].per_member;
  const int member = local / per, tile = local - member * per;
  const InstPtrs &ip = groups[gi].tab[member];
  if (ip.flags[0]) return;
  xpencil_body<T, NT, SC>(static_cast<cx<T> *>(ip.spec), A, gt, ip.aux, ip.ppart, tile);
}

// ------------------------------------------------------------ reduction
// Neumaier-compensated FP64 sums: each thread folds a strided share of the
// partials into (sum, compensation) pairs; the pairs are merged by a fixed
// shuffle tree within each warp and then across warps, so the result does
// not depend on timing.
__device__ __forceinline__ void neu_add(double &s, double &c, double v) {
  const double t = s + v;
  c += (fabs(s) >= fabs(v)) ? (s - t) + v : (v - t) + s;
  s = t;
}
__device__ __forceinline__ void neu_merge(double &s, double &c, double s2, double c2) {
  neu_add(s, c, s2);
  c += c2;
}
// merge (s0, c0), (s1, c1) over the block; thread 0 ends with the totals.
// scratch: 4 * 32 doubles.
__device__ __forceinline__ void block_neumaier2(double &s0, double &c0, double &s1, double &c1, double *scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double a = __shfl_down_sync(0xffffffffu, s0, o), b = __shfl_down_sync(0xffffffffu, c0, o);
    const double d = __shfl_down_sync(0xffffffffu, s1, o), e = __shfl_down_sync(0xffffffffu, c1, o);
    neu_merge(s0, c0, a, b);
    neu_merge(s1, c1, d, e);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) {
    scratch[wid] = s0; scratch[32 + wid] = c0; scratch[64 + wid] = s1; scratch[96 + wid] = c1;
  }
  __syncthreads();
  if (wid == 0) {
    s0 = lane < nw ? scratch[lane] : 0.0;
    c0 = lane < nw ? scratch[32 + lane] : 0.0;
    s1 = lane < nw ? scratch[64 + lane] : 0.0;
    c1 = lane < nw ? scratch[96 + lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double a = __shfl_down_sync(0xffffffffu, s0, o), b = __shfl_down_sync(0xffffffffu, c0, o);
      const double d = __shfl_down_sync(0xffffffffu, s1, o), e = __shfl_down_sync(0xffffffffu, c1, o);
      neu_merge(s0, c0, a, b);
      neu_merge(s1, c1, d, e);
    }
  }
}

// One block: stats[step] = {xinorm, xiave} from the per-plane partials (and
// the x-pencil partials of the Nyquist carrier, scaled); sets *stop when
// 0 < tol and xinorm < tol; flags a non-finite result in *bad.
static __global__ void k_finalize(const double *__restrict__ partials, int nparts, double *__restrict__ stats, int step,
                                  double tol, int *stop, int *bad, int *steps_done, const double *__restrict__ partials2,
                                  int nparts2, double scale2) {
  if (stop && *stop) return;
  __shared__ double sh[128];
  double s0 = 0, c0 = 0, s1 = 0, c1 = 0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    neu_add(s0, c0, partials[2 * i]);
    neu_add(s1, c1, partials[2 * i + 1]);
  }
  for (int i = threadIdx.x; i < nparts2; i += blockDim.x) neu_add(s0, c0, partials2[2 * i] * scale2);
  block_neumaier2(s0, c0, s1, c1, sh);
  if (threadIdx.x == 0) {
    const double xinorm = sqrt(s0 + c0), xiave = s1 + c1;
    stats[2 * step] = xinorm;
    stats[2 * step + 1] = xiave;
    if (steps_done) *steps_done = step + 1;
    if (!isfinite(xinorm) || !isfinite(xiave)) *bad = 1;
    if (tol > 0.0 && xinorm < tol && stop) *stop = 1;
  }
}

// One block per instance of a group: records {xinorm, xiave} at index
// flags[2] (when within the stats capacity), advances flags[2], flips the
// buffer parity flags[4], flags non-finite results and sets the stop flag
// when 0 < tol and xinorm < tol.
static __global__ void k_finalize_tab(const InstPtrs *__restrict__ tab, int nparts, int nparts2, double scale2,
                                      double tol) {
  const InstPtrs &ip = tab[blockIdx.x];
  int *flags = ip.flags;
  if (flags[0]) return;
  __shared__ double sh[128];
  const double *partials = ip.partials, *partials2 = ip.ppart;
  double s0 = 0, c0 = 0, s1 = 0, c1 = 0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    neu_add(s0, c0, partials[2 * i]);
    neu_add(s1, c1, partials[2 * i + 1]);
  }
  if (partials2)
    for (int i = threadIdx.x; i < nparts2; i += blockDim.x) neu_add(s0, c0, partials2[2 * i] * scale2);
  block_neumaier2(s0, c0, s1, c1, sh);
  if (threadIdx.x == 0) {
    const double xinorm = sqrt(s0 + c0), xiave = s1 + c1;
    const int k = flags[2];
    if (k < ip.stats_cap) {
      ip.stats[2 * k] = xinorm;
      ip.stats[2 * k + 1] = xiave;
    }
    flags[2] = k + 1;
    flags[4] ^= 1;
    if (!isfinite(xinorm) || !isfinite(xiave)) flags[1] = 1;
    if (tol > 0.0 && xinorm < tol) flags[0] = 1;
  }
}

// k_finalize_tab for every instance of a merge class: blockIdx.x runs over
// the instances of the groups in order (MultiLaunch::starts counts instances).
static __global__ void k_finalize_multi(const MultiFinalGroup *__restrict__ groups, MultiLaunch m, double tol) {
  const int gi = group_of_block(m);
  const MultiFinalGroup &G = groups[gi];
  const InstPtrs &ip = G.tab[blockIdx.x - m.starts[gi]];
  int *flags = ip.flags;
  if (flags[0]) return;
  __shared__ double sh[128];
  const double *partials = ip.partials, *partials2 = ip.ppart;
  double s0 = 0, c0 = 0, s1 = 0, c1 = 0;
  for (int i = threadIdx.x; i < G.nparts; i += blockDim.x) {
    neu_add(s0, c0, partials[2 * i]);
    neu_add(s1, c1, partials[2 * i + 1]);
  }
  if (partials2)
    for (int i = threadIdx.x; i < G.nparts2; i += blockDim.x) neu_add(s0, c0, partials2[2 * i] * G.scale2);
  block_neumaier2(s0, c0, s1, c1, sh);
  if (threadIdx.x == 0) {
    const double xinorm = sqrt(s0 + c0), xiave = s1 + c1;
    const int k = flags[2];
    if (k < ip.stats_cap) {
      ip.stats[2 * k] = xinorm;
      ip.stats[2 * k + 1] = xiave;
    }
    flags[2] = k + 1;
    flags[4] ^= 1;
    if (!isfinite(xinorm) || !isfinite(xiave)) flags[1] = 1;
    if (tol > 0.0 && xinorm < tol) flags[0] = 1;
  }
}

// ------------------------------------------------------------ stress state
// sigma_rot and tau in FP64 exactly as rotate_stress + resolSS_Schmid
// (fft_fftw_slab.cpp:242-274, 737-769); then optionally sigma += dsigma
// (solve_GL.cpp:151-155) and clear the stop flag.
// project_core_energy (fft_fftw_slab.cpp:1572-1595): delta of planes 0..np-1
// in FP64, Re xi_p for S <= 2, else the projection of systems 3p..3p+2 on b_1
// in the reference's order of operations.
struct ProfileArgs {
  double xb[3][3];
};

template <typename T>
static __global__ void k_core_profile(const T *__restrict__ xi, int S, size_t N, int np, ProfileArgs pa,
                                      double *__restrict__ delta) {
  const size_t total = (size_t)np * N;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const size_t p = q / N, r = q - p * N;
    if (S <= 2) {
      delta[q] = (double)xi[q];
    } else {
      const double x0 = (double)xi[(3 * p) * N + r], x1 = (double)xi[(3 * p + 1) * N + r],
                   x2 = (double)xi[(3 * p + 2) * N + r];
      double v = 0.0;
      for (int c = 0; c < 3; ++c)
        v = __dadd_rn(v, __dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(x0, pa.xb[0][c]), __dmul_rn(x1, pa.xb[1][c])),
                                             __dmul_rn(x2, pa.xb[2][c])),
                                   pa.xb[1][c]));
      delta[q] = v;
    }
  }
}

struct StressArgs {
  double prim[3][3], invprim[3][3];
  int ortho;
  int S;
  double xn[PFDD_MAXS][3], xb[PFDD_MAXS][3];
  double dslip;
  double dsig[3][3];
  int ns;                          // 1: tau from the non-Schmid projections proj
  double proj[PFDD_MAXS][3][3];    // S_tot[a][i][j] of resolSS_non_Schmid
  int usfe;                        // 1: core model 6 amplitude from sigma_rot[2][1]
  double fit[5];                   // a_slope, a_b, b_b, c_slope, c_b
  double fit_sin;                  // sin(b_b angle_to_110 pi / 180)
  double mu, s;                    // Material::mu, mu dslip b
};

// tau_a from sigma_rot: resolSS_Schmid (fft_fftw_slab.cpp:744-749) or
// resolSS_non_Schmid (:812-827), in the reference's order of operations; the
// core model 6 amplitude (core_energy_USFE_angle_tau :1517-1528) into an[]:
// an[0] = An' pi, an[1] = An', and the same two as floats after them.
__device__ __forceinline__ void resolve_state(const StressArgs &s, const double (&sr)[3][3], double *tau, double *an) {
  for (int a = 0; a < s.S; ++a) {
    double t = 0.0;
    if (s.ns) {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t = t + __ddiv_rn(__dmul_rn(sr[i][j], s.proj[a][i][j]), s.dslip);
    } else {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t = t + (sr[i][j] * s.xn[a][j] * s.xb[a][i]) / s.dslip;
    }
    tau[a] = t;
  }
  if (s.usfe && an) {
    const double m9 = 1.0E-9;
    const double ga = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(s.fit[0], sr[2][1]), s.mu), m9), s.fit[1]);
    const double gc = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(s.fit[3], sr[2][1]), s.mu), m9), s.fit[4]);
    const double gsfe = __dmul_rn(__dadd_rn(__dmul_rn(ga, s.fit_sin), gc), 1.0E-3);
    const double A = __ddiv_rn(gsfe, s.s);
    an[0] = __dmul_rn(A, PFDD_PI_T);
    an[1] = A;
    float *af = reinterpret_cast<float *>(an + 2);
    af[0] = (float)an[0];
    af[1] = (float)A;
  }
}

static __global__ void k_stress_state(double *sigma /*[9]*/, double *tau, double *an, StressArgs s, int mode, int *stop) {
  if (threadIdx.x != 0) return;
  if (mode == 0) {
    double sr[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        sr[i][j] = 0.0;
        if (s.ortho) {
          for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) sr[i][j] += s.prim[i][k] * sigma[3 * k + l] * s.invprim[l][j];
        } else {
          sr[i][j] = sigma[3 * i + j];
        }
      }
    resolve_state(s, sr, tau, an);
    if (stop) *stop = 0;
  } else {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) sigma[3 * i + j] = sigma[3 * i + j] + s.dsig[i][j];
  }
}

// One block per instance: mode 0 = sigma_rot and tau from the current sigma,
// clear the stop flag; mode 1 = sigma += dsigma (stored after sigma).
static __global__ void k_stress_state_tab(const InstPtrs *__restrict__ tab, StressArgs s, int mode) {
  if (threadIdx.x != 0) return;
  const InstPtrs &ip = tab[blockIdx.x];
  double *sigma = ip.sigma;
  if (mode == 0) {
    double sr[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        sr[i][j] = 0.0;
        if (s.ortho) {
          for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) sr[i][j] += s.prim[i][k] * sigma[3 * k + l] * s.invprim[l][j];
        } else {
          sr[i][j] = sigma[3 * i + j];
        }
      }
    resolve_state(s, sr, ip.tau, ip.an);
    ip.flags[0] = 0;
  } else {
    for (int i = 0; i < 9; ++i) sigma[i] = sigma[i] + sigma[9 + i];
  }
}

// ------------------------------------------------------------ adjoint reductions
// acc[0..1] += sums of the per-plane parameter partials over the real-field
// planes, acc[2 + a] += sum of lambda over system a's planes (each partial
// already summed over the backward steps by the plane passes); comp[] holds
// the Neumaier compensation terms.
static __global__ void k_grad_accum(const double *__restrict__ gpart, int S, int nx, double *acc, double *comp) {
  const int t = threadIdx.x;
  if (t >= 2 + S) return;
  double s = 0.0, c = 0.0;
  const int col = t < 2 ? t : 2;
  const int p0 = t < 2 ? 0 : (t - 2) * nx, p1 = t < 2 ? S * nx : (t - 1) * nx;
  for (int p = p0; p < p1; ++p) {
    const double v = gpart[4 * p + col], u = s + v;
    c += (fabs(s) >= fabs(v)) ? (s - u) + v : (v - u) + s;
    s = u;
  }
  const double v = s + c, u = acc[t] + v;
  comp[t] += (fabs(acc[t]) >= fabs(v)) ? (acc[t] - u) + v : (v - u) + acc[t];
  acc[t] = u;
}

// ------------------------------------------------------------ strain / stress diagnostics
// The strain field of the current state as FFTW_Slab::strain computes it with
// Fmatrix (fft_fftw_slab.cpp:644-732, 3370-3469):
//   strain_ij(k) = sum_s F[s,i,j](k) Z_s(k),  F[s,i,j] = k_i (G sigma^s k)_j,
//   G = (2 I / k^2 - k k^T / ((1 - nu) k^4)) / (2 mu)   (Voigt mu and nu),
// i.e. with Sig = sum_s sigma^s Z_s and U = Sig k:  strain = k w^T, w = G U,
// of which the diagnostics keep the symmetric part (data_eps).  Its real part
// follows the Im-carrier rule of the contraction: F(k) Xr off the Nyquist
// planes, (F(k)(Xr + i Xi) + F(k')(Xr - i Xi)) / 2 on them (or everywhere
// with the full carrier), k' the reference's vector of index -k.
template <typename T, typename C>
__device__ __forceinline__ void strain_of(const C (&sig)[6], T kx, T ky, T kz, T c1nu, T inv2mu, C (&o)[6]) {
  const T k2 = kx * kx + ky * ky + kz * kz;
  if (!(k2 > (T)0)) {
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = mk<C>((T)0, (T)0);
    return;
  }
  const T ik2 = (T)1 / k2;
  const C U0 = mk<C>(sig[0].x * kx + sig[3].x * ky + sig[4].x * kz, sig[0].y * kx + sig[3].y * ky + sig[4].y * kz);
  const C U1 = mk<C>(sig[3].x * kx + sig[1].x * ky + sig[5].x * kz, sig[3].y * kx + sig[1].y * ky + sig[5].y * kz);
  const C U2 = mk<C>(sig[4].x * kx + sig[5].x * ky + sig[2].x * kz, sig[4].y * kx + sig[5].y * ky + sig[2].y * kz);
  const C kU = mk<C>(kx * U0.x + ky * U1.x + kz * U2.x, kx * U0.y + ky * U1.y + kz * U2.y);
  const T a = (T)2 * ik2 * inv2mu, b = c1nu * ik2 * ik2 * inv2mu;
  const C w0 = mk<C>(a * U0.x - b * kx * kU.x, a * U0.y - b * kx * kU.y);
  const C w1 = mk<C>(a * U1.x - b * ky * kU.x, a * U1.y - b * ky * kU.y);
  const C w2 = mk<C>(a * U2.x - b * kz * kU.x, a * U2.y - b * kz * kU.y);
  const T h = (T)0.5;
  o[0] = mk<C>(kx * w0.x, kx * w0.y);
  o[1] = mk<C>(ky * w1.x, ky * w1.y);
  o[2] = mk<C>(kz * w2.x, kz * w2.y);
  o[3] = mk<C>(h * (kx * w1.x + ky * w0.x), h * (kx * w1.y + ky * w0.y));
  o[4] = mk<C>(h * (kx * w2.x + kz * w0.x), h * (kx * w2.y + kz * w0.y));
  o[5] = mk<C>(h * (ky * w2.x + kz * w1.x), h * (ky * w2.y + kz * w1.y));
}

// x pencils of the current state's half spectrum (F fields in) -> the six
// symmetric strain components (xx yy zz xy xz yz) after the inverse x FFT.
// grid.x = ncols / ccols; smem = (max(F, 6) * fstride + nx) * sizeof(C).
template <typename T, int NT>
__global__ void __launch_bounds__(NT, 2) k_strain_pencil(const cx<T> *__restrict__ spec, cx<T> *__restrict__ out6,
                                                         PencilArgs a) {
  using C = cx<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nx = a.nx, F = a.F, cc = a.ccols, S = a.S, fst = a.fstride;
  const int FB = F > 6 ? F : 6;
  C *buf = reinterpret_cast<C *>(smem_raw);
  C *twx = buf + (size_t)FB * fst;
  const size_t col0 = (size_t)blockIdx.x * cc, ncols = a.ncols;
  const int per = nx * cc;
  // (field, x) rows of the tile in 16-byte chunks (cp.async, as the x-pencil
  // pass) when a row is whole chunks; element by element otherwise
  const int cpr = (int)(cc * sizeof(C) / 16);
  const bool chunks = cpr > 0 && (cc * sizeof(C)) % 16 == 0;
  if (chunks) {
    for (int q = threadIdx.x; q < F * nx * cpr; q += blockDim.x) {
      const int fx = a.fd_cpr.div(q), ch = q - fx * cpr;
      const int f = a.fd_nx.div(fx), x = fx - f * nx;
      cp_async16(reinterpret_cast<char *>(buf + (size_t)f * fst + (size_t)x * cc) + 16 * ch,
                 reinterpret_cast<const char *>(spec + (size_t)fx * ncols + col0) + 16 * ch);
    }
  } else {
    for (int f = 0; f < F; ++f)
      for (int rem = threadIdx.x; rem < per; rem += blockDim.x) {
        const int x = a.fd_cc.div(rem), c = rem - x * cc;
        buf[(size_t)f * fst + (size_t)x * cc + c] = spec[((size_t)f * nx + x) * ncols + col0 + c];
      }
  }
  load_table(twx, a.tw_x, nx);
  if (chunks) cp_async_wait_all();
  __syncthreads();
  Batch gx{F * cc, cc, 1, fst, cc, true, a.fd_fcc, a.fd_cc};
  fft_forward<MaxRadix<NT>::value, GeomPencil>(buf, twx, a.px, gx);
  const GreenT<T> &g = green_t<T>(a.g);
  const C *caux = reinterpret_cast<const C *>(a.aux);
  const T c1nu = g.c1nu, inv2mu = (T)a.inv2mu;
  for (int w = threadIdx.x; w < per; w += blockDim.x) {
    const int sx = a.fd_cc.div(w), c = w - sx * cc;
    const int col = (int)(col0 + c);
    const int sy = a.fd_nzp.div(col), sz = col - sy * a.nzp;
    C *pk = buf + (size_t)sx * cc + c;
    C o[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = mk<C>((T)0, (T)0);
    if (sz <= a.M) {
      const int ix = a.kx_of[sx], iy = a.ky_of[sy], iz = a.kz_of[sz];
      const T fx = freq_of<T>(ix, a.nx), fy = freq_of<T>(iy, a.ny), fz = freq_of<T>(iz, a.nz);
      const T kx = fx * g.four[0][0] + fy * g.four[1][0] + fz * g.four[2][0];
      const T ky = fx * g.four[0][1] + fy * g.four[1][1] + fz * g.four[2][1];
      const T kz = fx * g.four[0][2] + fy * g.four[1][2] + fz * g.four[2][2];
      C sr[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) sr[q] = mk<C>((T)0, (T)0);
      for (int b = 0; b < S; ++b) green_accumulate<T>(g, b, pk[(size_t)b * fst], sr);
      bool nyq = false;
      size_t a0 = 0, astride = 0;
      if (a.imag == IMAG_NYQ) {
        a0 = nyq_index<T, C>(a, 0, sx, sy, sz, nyq);
        astride = (sz == a.M) ? (size_t)a.nx * a.ny : (sy == a.sy_n ? (size_t)a.nx * a.M : (size_t)a.ny * a.M);
      }
      if (a.imag == IMAG_FULL || nyq) {
        C si[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) si[q] = mk<C>((T)0, (T)0);
        for (int b = 0; b < S; ++b) {
          C y;
          if (a.imag == IMAG_FULL) y = pk[(size_t)(S + b) * fst];
          else y = caux[a0 + b * astride];
          green_accumulate<T>(g, b, y, si);
        }
        C sp[6], sq[6], op[6], oq[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          sp[q] = mk<C>(sr[q].x - si[q].y, sr[q].y + si[q].x);
          sq[q] = mk<C>(sr[q].x + si[q].y, sr[q].y - si[q].x);
        }
        const T gxn = freq_neg<T>(ix, a.nx), gyn = freq_neg<T>(iy, a.ny), gzn = freq_neg<T>(iz, a.nz);
        const T mx = gxn * g.four[0][0] + gyn * g.four[1][0] + gzn * g.four[2][0];
        const T my = gxn * g.four[0][1] + gyn * g.four[1][1] + gzn * g.four[2][1];
        const T mz = gxn * g.four[0][2] + gyn * g.four[1][2] + gzn * g.four[2][2];
        strain_of<T>(sp, kx, ky, kz, c1nu, inv2mu, op);
        strain_of<T>(sq, mx, my, mz, c1nu, inv2mu, oq);
#pragma unroll
        for (int q = 0; q < 6; ++q) o[q] = mk<C>((T)0.5 * (op[q].x + oq[q].x), (T)0.5 * (op[q].y + oq[q].y));
      } else {
        strain_of<T>(sr, kx, ky, kz, c1nu, inv2mu, o);
      }
    }
    // every input of this point has been read: its six outputs take slots 0..5
#pragma unroll
    for (int q = 0; q < 6; ++q) pk[(size_t)q * fst] = o[q];
  }
  __syncthreads();
  Batch g6{6 * cc, cc, 1, fst, cc, true, a.fd_6cc, a.fd_cc};
  fft_inverse<MaxRadix<NT>::value, GeomPencil>(buf, twx, a.px, g6);
  if (chunks) {
    for (int q = threadIdx.x; q < 6 * nx * cpr; q += blockDim.x) {
      const int fx = a.fd_cpr.div(q), ch = q - fx * cpr;
      const int f = a.fd_nx.div(fx), x = fx - f * nx;
      *reinterpret_cast<float4 *>(reinterpret_cast<char *>(out6 + (size_t)fx * ncols + col0) + 16 * ch) =
          *reinterpret_cast<const float4 *>(reinterpret_cast<const char *>(buf + (size_t)f * fst + (size_t)x * cc) +
                                            16 * ch);
    }
    return;
  }
  for (int f = 0; f < 6; ++f)
    for (int rem = threadIdx.x; rem < per; rem += blockDim.x) {
      const int x = a.fd_cc.div(rem), c = rem - x * cc;
      out6[((size_t)f * nx + x) * ncols + col0 + c] = buf[(size_t)f * fst + (size_t)x * cc + c];
    }
}

// ------------------------------------------------------------ conductivity
// divcurrent's two operators on the conductivity field c = X + iY (X, Y the
// spectra of Re and Im condxi, fft_fftw_slab.cpp:1699-1741): a = i (k_y/k^2) c
// and b = (k_y^2/k^2) c, zero at k = 0.  The reference's complex transforms
// index -k with its own frequency table (k' differs from -k on the Nyquist
// planes), so the spectra of the real and imaginary parts of each output are
//   Re: (M(k)(X+iY) + conj M'(X-iY)) / 2,   Im: (M(k)(X+iY) - conj M'(X-iY)) / 2i
// with M' the operator at k'.  Slots 0..3 out: Re a, Im a, Re b, Im b.
template <typename T, typename C>
__device__ __forceinline__ void cond_point(C x, C y, T ky, T k2, T kyn, T k2n, C (&o)[4]) {
  // M(k) c with c = X + iY
  const C c = mk<C>(x.x - y.y, x.y + y.x);
  const C d = mk<C>(x.x + y.y, x.y - y.x);   // X - iY
  const T ra = ky / k2, rb = ky * ky / k2;    // a: i ra c ; b: rb c
  const T rna = kyn / k2n, rnb = kyn * kyn / k2n;
  // a: p = i ra c, q = conj(i rna) d = -i rna d
  const C pa = mk<C>(-ra * c.y, ra * c.x), qa = mk<C>(rna * d.y, -rna * d.x);
  const C pb = mk<C>(rb * c.x, rb * c.y), qb = mk<C>(rnb * d.x, rnb * d.y);
  const T h = (T)0.5;
  o[0] = mk<C>(h * (pa.x + qa.x), h * (pa.y + qa.y));
  o[1] = mk<C>(h * (pa.y - qa.y), -h * (pa.x - qa.x));   // (p - q) / 2i
  o[2] = mk<C>(h * (pb.x + qb.x), h * (pb.y + qb.y));
  o[3] = mk<C>(h * (pb.y - qb.y), -h * (pb.x - qb.x));
}

// Per tile of (ky, kz) columns: x FFT of the two fields of condxi's spectrum,
// the four output spectra per point, inverse x FFT of the four.
template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_cond_pencil(const cx<T> *__restrict__ spec, cx<T> *__restrict__ out4,
                                                       PencilArgs a) {
  using C = cx<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nx = a.nx, cc = a.ccols, fst = a.fstride;
  C *buf = reinterpret_cast<C *>(smem_raw);   // [4][fstride]
  C *twx = buf + (size_t)4 * fst;
  const size_t col0 = (size_t)blockIdx.x * cc, ncols = a.ncols;
  const int per = nx * cc;
  for (int i = threadIdx.x; i < 2 * per; i += blockDim.x) {
    const int f = i / per, rem = i - f * per, x = rem / cc, c = rem - x * cc;
    buf[(size_t)f * fst + rem] = spec[((size_t)f * nx + x) * ncols + col0 + c];
  }
  load_table(twx, a.tw_x, nx);
  __syncthreads();
  Batch gx{2 * cc, cc, 1, fst, cc, true, a.fd_fcc, a.fd_cc};
  fft_forward<MaxRadix<NT>::value, GeomPencil>(buf, twx, a.px, gx);
  const GreenT<T> &g = green_t<T>(a.g);
  for (int w = threadIdx.x; w < per; w += blockDim.x) {
    const int sx = a.fd_cc.div(w), c = w - sx * cc;
    const int col = (int)(col0 + c);
    const int sy = a.fd_nzp.div(col), sz = col - sy * a.nzp;
    C *pk = buf + sx * cc + c;
    C o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = mk<C>((T)0, (T)0);
    if (sz <= a.M) {
      const int ix = a.kx_of[sx], iy = a.ky_of[sy], iz = a.kz_of[sz];
      const T fx = freq_of<T>(ix, a.nx), fy = freq_of<T>(iy, a.ny), fz = freq_of<T>(iz, a.nz);
      const T kx = fx * g.four[0][0] + fy * g.four[1][0] + fz * g.four[2][0];
      const T ky = fx * g.four[0][1] + fy * g.four[1][1] + fz * g.four[2][1];
      const T kz = fx * g.four[0][2] + fy * g.four[1][2] + fz * g.four[2][2];
      const T k2 = kx * kx + ky * ky + kz * kz;
      if (k2 > (T)0) {
        const T gxn = freq_neg<T>(ix, a.nx), gyn = freq_neg<T>(iy, a.ny), gzn = freq_neg<T>(iz, a.nz);
        const T mx = gxn * g.four[0][0] + gyn * g.four[1][0] + gzn * g.four[2][0];
        const T my = gxn * g.four[0][1] + gyn * g.four[1][1] + gzn * g.four[2][1];
        const T mz = gxn * g.four[0][2] + gyn * g.four[1][2] + gzn * g.four[2][2];
        cond_point<T, C>(pk[0], pk[(size_t)fst], ky, k2, my, mx * mx + my * my + mz * mz, o);
      }
    }
    // both inputs of this point have been read: its four outputs take slots 0..3
#pragma unroll
    for (int q = 0; q < 4; ++q) pk[(size_t)q * fst] = o[q];
  }
  __syncthreads();
  Batch g4{4 * cc, cc, 1, fst, cc, true, a.fd_6cc, a.fd_cc};
  fft_inverse<MaxRadix<NT>::value, GeomPencil>(buf, twx, a.px, g4);
  for (int i = threadIdx.x; i < 4 * per; i += blockDim.x) {
    const int f = i / per, rem = i - f * per, x = rem / cc, c = rem - x * cc;
    out4[((size_t)f * nx + x) * ncols + col0 + c] = buf[(size_t)f * fst + rem];
  }
}

// backwardcond's real-space assembly and update_conduct_order_param
// (fft_fftw_slab.cpp:2157-2186, 1816-1829) per site, in FP64: fr holds the
// unnormalised inverse transforms Re a, Im a, Re b, Im b; tab the effective
// conductivity [ny] and the y-derivative of the layer conductivity [ny].
// part[blk * 3 + {0,1,2}] = sum |dcondxi|^2, sum Re condxi, sum j_y / N.
struct CondArgs {
  double El, eps0, dt;
  int ny, nz;
};

template <typename T>
__global__ void k_cond_update(T *__restrict__ cxi, const T *__restrict__ fr, const double *__restrict__ tab,
                              CondArgs c, size_t N, double *__restrict__ part) {
  __shared__ double red[3 * 32];
  double v[3] = {0.0, 0.0, 0.0};
  const double nsz = (double)N, kdt = 1e-22 * c.dt;
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)((r / (size_t)c.nz) % (size_t)c.ny);
    const double cs = tab[j], dcs = tab[c.ny + j];
    const double jr = (double)fr[r], ji = (double)fr[N + r], br = (double)fr[2 * N + r], bi = (double)fr[3 * N + r];
    const double jcur = cs * (c.El - jr / c.eps0);
    v[2] += jcur / nsz;
    const double cre = (cs / c.eps0) * br + (jr / c.eps0 - c.El) * dcs;
    const double cim = (cs / c.eps0) * bi + (ji / c.eps0) * dcs;
    const double xr = (double)cxi[r], xi = (double)cxi[N + r];
    const T nr = (T)(xr - kdt * (cre / nsz)), ni = (T)(xi - kdt * (cim / nsz));
    cxi[r] = nr;
    cxi[N + r] = ni;
    const double dr = (double)nr - xr, di = (double)ni - xi;
    v[0] += dr * dr + di * di;
    v[1] += (double)nr;
  }
  block_reduce<3>(v, red);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = v[0];
    part[3 * blockIdx.x + 1] = v[1];
    part[3 * blockIdx.x + 2] = v[2];
  }
}

// Per-system sums of Re xi ([S][N], compute precision) in FP64: part[blk * S + s].
template <typename T>
__global__ void k_field_sums(const T *__restrict__ xr, int S, size_t N, double *__restrict__ part) {
  // 16-byte loads (N is a multiple of 4: nx and ny are even), one FP64
  // accumulator per vector lane, several loads in flight per thread
  using V = typename Vec<T>::type;
  constexpr int VN = Vec<T>::n;
  __shared__ double red[64];
  const size_t nv = N / VN, stride = (size_t)gridDim.x * blockDim.x;
  for (int s0 = 0; s0 < S; ++s0) {
    const V *p = reinterpret_cast<const V *>(xr + (size_t)s0 * N);
    double a[VN];
#pragma unroll
    for (int q = 0; q < VN; ++q) a[q] = 0.0;
#pragma unroll 4
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nv; i += stride) {
      T t[VN];
      *reinterpret_cast<V *>(t) = p[i];
#pragma unroll
      for (int q = 0; q < VN; ++q) a[q] += (double)t[q];
    }
    double acc = a[0];
#pragma unroll
    for (int q = 1; q < VN; ++q) acc += a[q];
    double out[2];
    block_sum2(acc, 0.0, red, out);
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * S + s0] = out[0];
    __syncthreads();
  }
}

// Constants of the stress field (stress, fft_fftw_slab.cpp:3474-3553), FP64.
struct StressFieldArgs {
  double e6[PFDD_MAXS][6];   // sym(eps^s): xx yy zz xy xz yz
  double avepst6[6];         // sym(avepst) = sym(S : sigma_rot mu + <eps0>)
  double avepsts6[6];        // sym(S : sigma_rot mu)
  double sigmu[9];           // sigma_rot * mu, row major
  double C44, C12;
  int S;
};

// Per site: eps = strain + avepst (symmetric), eps0 = sum_s eps^s Re xi_s,
// X = eps - eps0 - avepsts, sigma = C : X + sigma_rot mu = 2 C44 X + C12 tr(X) I
// + sigma_rot mu (C isotropic, X symmetric).  Writes eps9 / sig9 ([3][3][N],
// FP64, either may be null) and per-block FP64 sums of their 18 components.
template <typename T>
__global__ void k_stress_fields(const T *__restrict__ strain6, const T *__restrict__ xr, size_t N,
                                StressFieldArgs p, double *__restrict__ eps9, double *__restrict__ sig9,
                                double *__restrict__ part) {
  __shared__ double red[18 * 32 + 18];
  double acc[18];
#pragma unroll
  for (int q = 0; q < 18; ++q) acc[q] = 0.0;
  const int map[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};   // (i, j) -> xx yy zz xy xz yz
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < N; r += (size_t)gridDim.x * blockDim.x) {
    double e[6], x[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) e[q] = (double)strain6[(size_t)q * N + r] + p.avepst6[q];
    double d[6] = {0, 0, 0, 0, 0, 0};
    for (int s0 = 0; s0 < p.S; ++s0) {
      const double v = (double)xr[(size_t)s0 * N + r];
#pragma unroll
      for (int q = 0; q < 6; ++q) d[q] += p.e6[s0][q] * v;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) x[q] = e[q] - d[q] - p.avepsts6[q];
    const double tr = x[0] + x[1] + x[2];
#pragma unroll
    for (int ij = 0; ij < 9; ++ij) {
      const int i = ij / 3, j = ij - 3 * i, q = map[ij];
      const double ev = e[q];
      const double sv = 2.0 * p.C44 * x[q] + (i == j ? p.C12 * tr : 0.0) + p.sigmu[ij];
      if (eps9) eps9[(size_t)ij * N + r] = ev;
      if (sig9) sig9[(size_t)ij * N + r] = sv;
      acc[ij] += ev;
      acc[9 + ij] += sv;
    }
  }
  plane_sum<false, 18>(acc, red, part + 18 * (size_t)blockIdx.x);
}

// ------------------------------------------------------------ layout helpers
template <typename T>
__global__ void k_from_interleaved(const double *__restrict__ src, T *__restrict__ re, T *__restrict__ im, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = reinterpret_cast<const double2 *>(src)[i];
    re[i] = (T)v.x;
    if (im) im[i] = (T)v.y;
  }
}

template <typename T>
__global__ void k_to_interleaved(const T *__restrict__ re, const T *__restrict__ im, double *__restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double2 v;
    v.x = (double)re[i];
    v.y = im ? (double)im[i] : 0.0;
    reinterpret_cast<double2 *>(dst)[i] = v;
  }
}

template <typename T>
__global__ void k_from_planar(const double *__restrict__ src, T *__restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (T)src[i];
}

template <typename T>
__global__ void k_to_planar(const T *__restrict__ src, double *__restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

}  // namespace pfdd
