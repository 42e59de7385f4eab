// Device FFT building blocks for the PFDD Ginzburg-Landau stepper (sm_100a).
//
// Transforms run in place in shared memory as a sequence of mixed-radix
// decimation-in-frequency stages (radices 2, 3, 4, 8, 16).  Stage s of a
// length-n transform has sub-length L_s (L_0 = n, L_{s+1} = L_s / R_s); work
// item (block, j) loads R_s elements at positions block*L_s + j + r*L_s/R_s,
// applies a register DFT of size R_s, multiplies output k by W_{L_s}^{j*k}
// and stores back to the same positions.  The forward transform therefore
// maps natural order to a digit-reversed order: frequency
//   k = k_0 + R_0 k_1 + R_0 R_1 k_2 + ...
// ends at position k_0 L_1 + k_1 L_2 + ... .  The inverse runs the stages in
// reverse with conjugate twiddles and the conjugate DFT, mapping the
// digit-reversed order back to natural order, unnormalised.  Consumers of the
// spectrum read frequencies through per-axis slot->k tables built on the host.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pfdd_fastdiv.h"

namespace pfdd {

template <typename T> struct cx_of;
template <> struct cx_of<float> { using type = float2; };
template <> struct cx_of<double> { using type = double2; };
template <typename T> using cx = typename cx_of<T>::type;

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r; r.x = a; r.y = b; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return mk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
#ifndef PFDD_NO_F32X2
// FP32 complex add / subtract as one packed f32x2 add (sm_100 FADD2; same
// rounding as two scalar adds).  A packed complex multiply measured slower
// (its operand shuffles cost more than the packing saves), so cmul stays scalar.
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
#endif
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { return mk<C>(a.x * s, a.y * s); }
// multiply by SIGN * i
template <int SIGN, typename C> __device__ __forceinline__ C mul_si(C a) {
  return mk<C>(-SIGN * a.y, SIGN * a.x);
}

// Exact constants (decimal expansions of cos/sin of multiples of pi/8, pi/3).
#define PFDD_H 0.70710678118654752440084436210484903928
#define PFDD_C8 0.92387953251128675612818318939678828682
#define PFDD_S8 0.38268343236508977172845998403039886676
#define PFDD_S3 0.86602540378443864676372317075293618347

// multiply by W_16^M = exp(SIGN * 2 pi i M / 16), M in 0..15
template <int M, int SIGN, typename C> __device__ __forceinline__ C tw16(C a) {
  using T = decltype(C::x);
  constexpr int m = M & 15;
  if constexpr (m == 0) return a;
  else if constexpr (m == 4) return mul_si<SIGN>(a);
  else if constexpr (m == 8) return mk<C>(-a.x, -a.y);
  else if constexpr (m == 12) return mul_si<-SIGN>(a);
  else {
    constexpr double cr[16] = {1, PFDD_C8, PFDD_H, PFDD_S8, 0, -PFDD_S8, -PFDD_H, -PFDD_C8,
                               -1, -PFDD_C8, -PFDD_H, -PFDD_S8, 0, PFDD_S8, PFDD_H, PFDD_C8};
    constexpr double sr[16] = {0, PFDD_S8, PFDD_H, PFDD_C8, 1, PFDD_C8, PFDD_H, PFDD_S8,
                               0, -PFDD_S8, -PFDD_H, -PFDD_C8, -1, -PFDD_C8, -PFDD_H, -PFDD_S8};
    const T wr = (T)cr[m], wi = (T)(SIGN * sr[m]);
    return mk<C>(a.x * wr - a.y * wi, a.x * wi + a.y * wr);
  }
}

template <int SIGN, typename C> __device__ __forceinline__ void dft2(C &a, C &b) {
  C t = a; a = cadd(t, b); b = csub(t, b);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft4(C &v0, C &v1, C &v2, C &v3) {
  C t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = mul_si<SIGN>(csub(v1, v3));
  v0 = cadd(t0, t2); v2 = csub(t0, t2); v1 = cadd(t1, t3); v3 = csub(t1, t3);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft3(C &v0, C &v1, C &v2) {
  using T = decltype(C::x);
  C s = cadd(v1, v2), d = csub(v1, v2);
  C m = mk<C>(v0.x - (T)0.5 * s.x, v0.y - (T)0.5 * s.y);
  const T s3 = (T)(SIGN * PFDD_S3);
  C isd = mk<C>(-s3 * d.y, s3 * d.x);
  v0 = cadd(v0, s);
  v1 = cadd(m, isd);
  v2 = csub(m, isd);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft8(C *v) {
  dft4<SIGN>(v[0], v[2], v[4], v[6]);
  dft4<SIGN>(v[1], v[3], v[5], v[7]);
  // odd outputs sit at v[1],v[3],v[5],v[7] for k = 0..3; twiddle by W8^k = W16^(2k)
  C o1 = tw16<2, SIGN>(v[3]), o2 = tw16<4, SIGN>(v[5]), o3 = tw16<6, SIGN>(v[7]);
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft16(C *v) {
  // n = 4 n1 + n2, k = k1 + 4 k2
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4<SIGN>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
  // v[4*k1 + n2] holds Y[n2][k1]; twiddle by W16^(n2*k1)
  v[5] = tw16<1, SIGN>(v[5]);  v[6] = tw16<2, SIGN>(v[6]);  v[7] = tw16<3, SIGN>(v[7]);
  v[9] = tw16<2, SIGN>(v[9]);  v[10] = tw16<4, SIGN>(v[10]); v[11] = tw16<6, SIGN>(v[11]);
  v[13] = tw16<3, SIGN>(v[13]); v[14] = tw16<6, SIGN>(v[14]); v[15] = tw16<9, SIGN>(v[15]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<SIGN>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // v[4*k1 + k2] holds X[k1 + 4 k2]; transpose to natural order
  C t[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = t[i];
}

template <int R, int SIGN, typename C> __device__ __forceinline__ void dft(C *v) {
  if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
  else if constexpr (R == 3) dft3<SIGN>(v[0], v[1], v[2]);
  else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 8) dft8<SIGN>(v);
  else if constexpr (R == 16) dft16<SIGN>(v);
}

// Radix plan of one axis, built on the host, with the per-stage divisors:
// stage s has n / R_s work items per transform (per[s]) and L_s / R_s
// positions j per block (lr[s]); its twiddles step by n / L_s (twstep[s]).
struct FftPlan {
  int n;
  int nst;
  int radix[8];
  int L[8];
  int twstep[8];
  FastDiv per[8], lr[8];
};

// Batched transform geometry in shared memory: transform b (0 <= b < batch)
// starts at (b % bin) * bs_in + (b / bin) * bs_out and its element i sits at
// start + i * es.  If batch_fast, consecutive threads take consecutive b (use
// when bs_in == 1); otherwise consecutive butterflies of one transform.
// fb and fi divide by batch and bin (built by the caller, outside the stages).
struct Batch {
  int batch, bin, bs_in, bs_out, es;
  bool batch_fast;
  FastDiv fb, fi;
};

// multiply v[k] (k = 1..R-1) by W^(j k) (or its conjugate), W^(j k) built from
// at most four table reads W^j, W^2j, W^4j, W^8j as the loop goes
// Twiddles W^(jk) read directly from the length-n table (measured faster than
// building them from W^j, W^2j, W^4j, W^8j by products: 0.5 % on 256x256x128,
// 3.5 % on 64^3 FP64; and each is a correctly rounded value, not a product).
#ifndef PFDD_TW_TABLE
#define PFDD_TW_TABLE 1
#endif
template <int R, bool CONJ, typename C>
__device__ __forceinline__ void apply_twiddles(C *v, const C *__restrict__ tw, int jt) {
  if constexpr (PFDD_TW_TABLE && R != 3) {
    // W^(jk) read directly: j k twstep < n, the table's length
#pragma unroll
    for (int k = 1; k < R; ++k) {
      const C w = tw[k * jt];
      v[k] = CONJ ? cmulc(v[k], w) : cmul(v[k], w);
    }
  } else if constexpr (R == 3) {
    const C w1 = tw[jt], w2 = tw[2 * jt];
    v[1] = CONJ ? cmulc(v[1], w1) : cmul(v[1], w1);
    v[2] = CONJ ? cmulc(v[2], w2) : cmul(v[2], w2);
  } else {
    C p[4];
#pragma unroll
    for (int b = 0; b < 4; ++b)
      if ((1 << b) < R) p[b] = tw[(1 << b) * jt];
#pragma unroll
    for (int k = 1; k < R; ++k) {
      // W^(jk) = product of W^(2^b j) over the set bits b of k
      C w;
      bool first = true;
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if (k & (1 << b)) {
          w = first ? p[b] : cmul(w, p[b]);
          first = false;
        }
      v[k] = CONJ ? cmulc(v[k], w) : cmul(v[k], w);
    }
  }
}

// Call-site geometry of a batched transform, fixed at compile time: BF (the
// batch_fast order), ES (element stride when known, 0 = Batch::es) and TWO_D
// (transform b starts at (b % bin) bs_in + (b / bin) bs_out; otherwise at
// b bs_in).
template <bool BF_, int ES_, bool TWO_D_> struct Geom {
  static constexpr bool BF = BF_;
  static constexpr int ES = ES_;
  static constexpr bool TWO_D = TWO_D_;
};
using GeomRows = Geom<false, 1, false>;   // contiguous rows, one transform per row
using GeomCols = Geom<true, 0, false>;    // columns of a row-major plane
using GeomPencil = Geom<true, 0, true>;   // columns of several fields

// The radix plan of make_plan (greedy 16, 8, 4, 2, 3 under MAXR) at compile
// time, for the lengths whose stages are specialised.
template <int N, int MAXR> struct SPlan {
  __host__ __device__ static constexpr int pick(int rem) {
    return (rem % 16 == 0 && MAXR >= 16) ? 16 : (rem % 8 == 0 && MAXR >= 8) ? 8 : (rem % 4 == 0) ? 4 :
           (rem % 2 == 0) ? 2 : 3;
  }
  __host__ __device__ static constexpr int len(int s) {   // L_s
    int rem = N;
    for (int i = 0; i < s; ++i) rem /= pick(rem);
    return rem;
  }
  __host__ __device__ static constexpr int radix(int s) { return pick(len(s)); }
  __host__ __device__ static constexpr int nst() {
    int rem = N, c = 0;
    while (rem > 1) { rem /= pick(rem); ++c; }
    return c;
  }
};

// One stage of radix R.  SL > 0: the stage length L = SL of a transform of
// length SN is known at compile time (index math folds to constants);
// otherwise L and the divisors come from the plan's stage s.
template <int R, bool INV, class G, int SN, int SL, typename C>
__device__ __forceinline__ void fft_stage(C *__restrict__ x, const C *__restrict__ tw, const FftPlan &p, int s,
                                          const Batch &g, int tid, int nthr) {
  constexpr bool ST = SL > 0;
  const int L = ST ? SL : p.L[s];
  const int Lr = L / R;
  const int per = ST ? SN / R : (int)p.per[s].d;
  constexpr int STW = ST ? SN / (ST ? SL : 1) : 0;   // twiddle step of a static stage
  const int twstep = ST ? STW : p.twstep[s];
  const int total = g.batch * per;
  const int es = G::ES ? G::ES : g.es;
  const int st = Lr * es;
  for (int w = tid; w < total; w += nthr) {
    int b, bf;
    if constexpr (G::BF) {
      bf = g.fb.div(w);
      b = w - bf * g.batch;
    } else if constexpr (ST) {
      b = w / per;
      bf = w - b * per;
    } else {
      b = p.per[s].div(w);
      bf = w - b * per;
    }
    int blk;
    if constexpr (ST) blk = bf / Lr;
    else blk = p.lr[s].div(bf);
    const int j = bf - blk * Lr;
    int off;
    if constexpr (G::TWO_D) {
      const int bq = g.fi.div(b);
      off = (b - bq * g.bin) * g.bs_in + bq * g.bs_out;
    } else {
      off = b * g.bs_in;
    }
    C *base = x + off + (blk * L + j) * es;
    C v[R];
    // contiguous elements (last stage along a unit-stride axis): 16-byte vectors
    constexpr bool VEC = sizeof(C) == 8 && (R % 2 == 0);
    const bool vec = VEC && st == 1;
    if (vec) {
#pragma unroll
      for (int r = 0; r < R; r += 2) {
        const float4 q = reinterpret_cast<const float4 *>(base)[r / 2];
        v[r] = mk<C>(q.x, q.y);
        v[r + 1] = mk<C>(q.z, q.w);
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = base[r * st];
    }
    if constexpr (!INV) {
      dft<R, -1>(v);
      if (j) apply_twiddles<R, false>(v, tw, j * twstep);
    } else {
      if (j) apply_twiddles<R, true>(v, tw, j * twstep);
      dft<R, 1>(v);
    }
    if (vec) {
#pragma unroll
      for (int r = 0; r < R; r += 2)
        reinterpret_cast<float4 *>(base)[r / 2] = make_float4(v[r].x, v[r].y, v[r + 1].x, v[r + 1].y);
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) base[r * st] = v[r];
    }
  }
}

// Radices above MAXR are compiled out (the host plans never use them for
// such a kernel), which bounds the registers a butterfly needs.
template <bool INV, int MAXR, class G, typename C>
__device__ __forceinline__ void fft_stage_dispatch(C *x, const C *tw, const FftPlan &p, int s, const Batch &g,
                                                   int tid, int nthr) {
  switch (p.radix[s]) {
    case 2: fft_stage<2, INV, G, 0, 0>(x, tw, p, s, g, tid, nthr); break;
    case 3: fft_stage<3, INV, G, 0, 0>(x, tw, p, s, g, tid, nthr); break;
    case 4: fft_stage<4, INV, G, 0, 0>(x, tw, p, s, g, tid, nthr); break;
    case 8: if constexpr (MAXR >= 8) fft_stage<8, INV, G, 0, 0>(x, tw, p, s, g, tid, nthr); break;
    case 16: if constexpr (MAXR >= 16) fft_stage<16, INV, G, 0, 0>(x, tw, p, s, g, tid, nthr); break;
    default: break;
  }
}

// Stages I.. of a length-N transform with the compile-time plan (forward in
// plan order, inverse in reverse), each followed by __syncthreads().
template <bool INV, int MAXR, class G, int N, int I> struct StaticStages {
  template <typename C> __device__ __forceinline__ static void run(C *x, const C *tw, const FftPlan &p, const Batch &g) {
    constexpr int NS = SPlan<N, MAXR>::nst();
    if constexpr (I < NS) {
      constexpr int s = INV ? NS - 1 - I : I;
      fft_stage<SPlan<N, MAXR>::radix(s), INV, G, N, SPlan<N, MAXR>::len(s)>(x, tw, p, s, g, threadIdx.x,
                                                                             blockDim.x);
      __syncthreads();
      StaticStages<INV, MAXR, G, N, I + 1>::run(x, tw, p, g);
    }
  }
};

// true when the host plan is the compile-time plan of length N
template <int N, int MAXR> __device__ __forceinline__ bool plan_is_static(const FftPlan &p) {
  if (p.n != N || p.nst != SPlan<N, MAXR>::nst()) return false;
  for (int s = 0; s < p.nst; ++s)
    if (p.radix[s] != SPlan<N, MAXR>::radix(s)) return false;
  return true;
}

// FP32 transforms of the common lengths run with compile-time plans (about
// 2% faster on 256x256x128); FP64 keeps the plan-driven loop, whose register
// footprint is smaller.
template <bool INV, int MAXR, class G, typename C>
__device__ __forceinline__ void fft_run(C *x, const C *tw, const FftPlan &p, const Batch &g) {
  if constexpr (sizeof(C) == 8) {
    if (plan_is_static<256, MAXR>(p)) { StaticStages<INV, MAXR, G, 256, 0>::run(x, tw, p, g); return; }
    if (plan_is_static<128, MAXR>(p)) { StaticStages<INV, MAXR, G, 128, 0>::run(x, tw, p, g); return; }
    if (plan_is_static<64, MAXR>(p)) { StaticStages<INV, MAXR, G, 64, 0>::run(x, tw, p, g); return; }
    if (plan_is_static<32, MAXR>(p)) { StaticStages<INV, MAXR, G, 32, 0>::run(x, tw, p, g); return; }
  }
  if constexpr (!INV) {
    for (int s = 0; s < p.nst; ++s) {
      fft_stage_dispatch<false, MAXR, G>(x, tw, p, s, g, threadIdx.x, blockDim.x);
      __syncthreads();
    }
  } else {
    for (int s = p.nst - 1; s >= 0; --s) {
      fft_stage_dispatch<true, MAXR, G>(x, tw, p, s, g, threadIdx.x, blockDim.x);
      __syncthreads();
    }
  }
}

// Forward (natural -> digit-reversed).  Ends with __syncthreads().
template <int MAXR, class G, typename C>
__device__ void fft_forward(C *x, const C *tw, const FftPlan &p, const Batch &g) {
  fft_run<false, MAXR, G>(x, tw, p, g);
}

// Inverse, unnormalised (digit-reversed -> natural).  Ends with __syncthreads().
template <int MAXR, class G, typename C>
__device__ void fft_inverse(C *x, const C *tw, const FftPlan &p, const Batch &g) {
  fft_run<true, MAXR, G>(x, tw, p, g);
}

// ------------------------------------------------------------ async copies
// Bulk (TMA) copies between global and shared memory with an mbarrier; every
// wait is bounded and reports a timeout instead of spinning forever.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Time limits of the bulk-copy waits: kWaitNs in normal operation (a copy of
// a few hundred KB lands within microseconds, so a second means the copy
// engine is gone), kStallWaitNs for the first wait when the stall test switch
// is on (a barrier that nothing completes; see plane_wait below).
constexpr uint64_t kWaitNs = 1000000000ull;
constexpr uint64_t kStallWaitNs = 200000ull;
// Returns false if the phase did not complete within limit_ns of %globaltimer.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns = kWaitNs) {
  const uint32_t a = smem_u32(bar);
  const uint32_t hint = limit_ns < 1000000ull ? (uint32_t)limit_ns : 1000000u;
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(hint)
        : "memory");
    if (done) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}
// Arrivals the plane passes' copy barrier expects: one (thread 0's
// arrive.expect_tx), plus one that nothing delivers while the stall test
// switch (err[2], an instance's flags[5]) is on.
__device__ __forceinline__ int stall_switch(const int *err) {
  return err ? *reinterpret_cast<const volatile int *>(err + 2) : 0;
}
// Wait of a plane-pass CTA for its bulk copies (phase 0 of bar).  Returns
// false after a timeout, with err[0] set; before returning it waits (bounded
// again) until the copies into this CTA's shared memory have landed: with the
// stall switch on, thread 0 delivers the withheld arrival so the phase
// completes exactly when the copies have.  Every thread of the CTA calls it.
__device__ __forceinline__ bool plane_wait(uint64_t *bar, int stall, int *err) {
  const bool ok = __syncthreads_and(mbar_wait(bar, 0, stall ? kStallWaitNs : kWaitNs));
  if (!ok) {
    if (threadIdx.x == 0) {
      if (stall) mbar_arrive(bar);
      if (err) atomicExch(err, 1);
    }
    __syncthreads();
    mbar_wait(bar, 0, kWaitNs);
    __syncthreads();
  }
  return ok;
}
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_s2g(void *dst_gmem, const void *src_smem, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
               "r"(smem_u32(src_smem)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// waits until the pending bulk stores have read their shared-memory source;
// the global writes complete before the grid does
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 16-byte asynchronous global->shared copy (cp.async), waited by cp_async_wait_all.
__device__ __forceinline__ void cp_async16(void *dst_smem, const void *src_gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst_smem)), "l"(src_gmem) : "memory");
}
// Bulk prefetch of a contiguous global range into L2 (16-byte aligned start
// and size); nothing waits for it.
__device__ __forceinline__ void prefetch_l2_bulk(const void *src_gmem, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src_gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

}  // namespace pfdd
