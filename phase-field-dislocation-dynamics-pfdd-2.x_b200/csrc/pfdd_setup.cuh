// Host-side FP64 set-up shared by the C-ABI entry points: radix plans and
// digit-reversal tables of the shared-memory FFTs, twiddle tables, and the
// per-instance constants of the Green's contraction, the GSFE core force and
// the stress state (what FFTW_Slab::setup computes in the reference,
// fft_fftw_slab.cpp:111-119).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "pfdd_b200.h"
#include "pfdd_kernels.cuh"

namespace pfdd {
namespace host {

// A kernel's dynamic shared-memory limit is one value per process and device,
// shared by every handle and by the allocation-free entry point: raise it to
// what a caller needs, never lower it under another caller's launches.
template <typename K>
inline cudaError_t raise_smem_limit(K *kernel, size_t bytes) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(kernel));
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(reinterpret_cast<const void *>(kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

// Radix plan: greedy 16, 8, 4, 2, 3 factors; sub-lengths L_s.
inline bool make_plan(int n, FftPlan &p, int maxr = 16) {
  p.n = n;
  p.nst = 0;
  int rem = n, L = n;
  while (rem > 1) {
    int r;
    if (rem % 16 == 0 && maxr >= 16) r = 16;
    else if (rem % 8 == 0 && maxr >= 8) r = 8;
    else if (rem % 4 == 0) r = 4;
    else if (rem % 2 == 0) r = 2;
    else if (rem % 3 == 0) r = 3;
    else return false;
    if (p.nst >= 8) return false;
    p.radix[p.nst] = r;
    p.L[p.nst] = L;
    p.twstep[p.nst] = n / L;
    p.per[p.nst] = FastDiv(n / r);
    p.lr[p.nst] = FastDiv(L / r);
    ++p.nst;
    L /= r;
    rem /= r;
  }
  return true;
}

// z plans (length M = nz/2 of the packed real rows): radix 8 then M/8 for
// M = 16, 32, 64, so that the register-resident z passes hold 8 complex
// values per thread in their middle pass; the greedy plan otherwise.  The
// kernels' ZPlan<M> follows the same rule.
inline bool make_zplan(int M, FftPlan &p, int maxr = 16) {
  if (!((M == 16 || M == 32 || M == 64) && maxr >= 8)) return make_plan(M, p, maxr);
  const int r2 = M / 8;
  p.n = M;
  p.nst = 2;
  p.radix[0] = 8;  p.L[0] = M;  p.twstep[0] = 1; p.per[0] = FastDiv(M / 8); p.lr[0] = FastDiv(M / 8);
  p.radix[1] = r2; p.L[1] = r2; p.twstep[1] = 8; p.per[1] = FastDiv(8);     p.lr[1] = FastDiv(1);
  return true;
}

// Host-built divisors of the plane and pencil kernels (after the integer
// fields of the argument block are set).
template <typename T> inline void set_plane_divisors(PlaneArgs &pa, int rows) {
  pa.fd_rows = FastDiv(rows);
  pa.fd_nvec = FastDiv(pa.nz / (sizeof(T) == 4 ? 4 : 2));
  pa.fd_m = FastDiv(pa.M);
  pa.fd_mh = FastDiv(pa.M / 2);
}
template <typename T> inline void set_pencil_divisors(PencilArgs &pe) {
  pe.fd_fcc = FastDiv(pe.F * pe.ccols);
  pe.fd_cc = FastDiv(pe.ccols);
  pe.fd_nzp = FastDiv(pe.nzp);
  pe.fd_cpr = FastDiv((int)(pe.ccols * sizeof(cx<T>) / 16));
  pe.fd_nx = FastDiv(pe.nx);
}

// Slot of -ky for every local y slot (PlaneArgs::negy).  pos[k] is the slot
// of frequency k under the y plan (length ny, or ny/2 for a split plane whose
// rank r holds ky = r + 2k at the slots of the ny/2 plan); rank r's entries
// start at r * (ny/2).  Stack storage only (ny <= 1024).
inline void neg_slots(int ny, bool split, const int *pos, int16_t *out) {
  const int n = split ? ny / 2 : ny;
  int kloc[1024];
  for (int k = 0; k < n; ++k) kloc[pos[k]] = k;
  for (int r = 0; r < (split ? 2 : 1); ++r)
    for (int sl = 0; sl < n; ++sl) {
      const int ky = split ? r + 2 * kloc[sl] : kloc[sl];
      const int nk = (ny - ky) % ny;   // same parity as ky (ny even)
      out[r * n + sl] = (int16_t)pos[split ? (nk - r) / 2 : nk];
    }
}

// k = 1..M/2 sorted by the slot pos[k] (PlaneArgs::kord), so consecutive
// threads of the (un)packing loops touch neighbouring slots.  Stack only.
inline void unpack_order(const int *pos, int M, int16_t *out) {
  const int mh = M / 2;
  for (int i = 0; i < mh; ++i) out[i] = (int16_t)(i + 1);
  for (int i = 1; i < mh; ++i)   // insertion sort by slot (M <= 512)
    for (int j = i; j > 0 && pos[out[j]] < pos[out[j - 1]]; --j) {
      const int16_t t = out[j];
      out[j] = out[j - 1];
      out[j - 1] = t;
    }
}

// position of frequency k after the forward (digit-reversing) transform
inline std::vector<int> positions(const FftPlan &p) {
  std::vector<int> pos(p.n);
  for (int k = 0; k < p.n; ++k) {
    int rem = k, q = 0;
    for (int s = 0; s < p.nst; ++s) {
      int d = rem % p.radix[s];
      rem /= p.radix[s];
      q += d * (p.L[s] / p.radix[s]);
    }
    pos[k] = q;
  }
  return pos;
}

// W_n^m = exp(-2 pi i m / n), m = 0..count-1, evaluated in FP64 with the
// angle reduced to the first octant's neighbourhood before cos/sin.
inline void twiddles(int n, int count, std::vector<double> &out) {
  out.resize(2 * (size_t)count);
  for (int m = 0; m < count; ++m) {
    long long e = m % n;
    double ang = 2.0 * M_PI * (double)e / (double)n;
    out[2 * m] = std::cos(ang);
    out[2 * m + 1] = -std::sin(ang);
  }
}

// Green constants in FP64: sigma^a = C44 (eps^a + eps^a^T) + C12 tr(eps^a) I,
// eps^a = xb_a (x) xn_a / dslip (fft_fftw_slab.cpp:559-566); mu and nu by the
// Voigt average (fft_fftw_slab.cpp:483-491).
inline void build_green(const pfdd_instance_desc &d, Green &g) {
  memset(&g, 0, sizeof g);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) g.four[i][j] = d.four[i][j];
  const double C44 = d.C44, C12 = d.C12, C11 = d.C11;
  const double mu = C44 - (2.0 * C44 + C12 - C11) / 5.0;
  const double ll = C12 - (2.0 * C44 + C12 - C11) / 5.0;
  const double young = mu * (3 * ll + 2 * mu) / (ll + mu);
  const double xnu = young / 2.0 / mu - 1.0;
  g.inv_mu = 1.0 / mu;
  g.c2 = 1.0 / (2.0 * C44);
  g.c1nu = 1.0 / (1.0 - xnu);
  for (int a = 0; a < d.n_slip; ++a) {
    double e[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) e[i][j] = d.xb[a][i] * d.xn[a][j] / d.dslip;
    const double tr = e[0][0] + e[1][1] + e[2][2];
    double s[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) s[i][j] = C44 * (e[i][j] + e[j][i]) + (i == j ? C12 * tr : 0.0);
    g.sig[a][0] = s[0][0]; g.sig[a][1] = s[1][1]; g.sig[a][2] = s[2][2];
    g.sig[a][3] = s[0][1]; g.sig[a][4] = s[0][2]; g.sig[a][5] = s[1][2];
    g.eps[a][0] = e[0][0]; g.eps[a][1] = e[1][1]; g.eps[a][2] = e[2][2];
    g.eps[a][3] = e[0][1] + e[1][0]; g.eps[a][4] = e[0][2] + e[2][0]; g.eps[a][5] = e[1][2] + e[2][1];
  }
  // per-precision tables: sigma for Sig, sigma/mu and eps/mu for the output
  auto fill = [&](auto &t) {
    using T = typename std::remove_reference<decltype(t.c2)>::type;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) t.four[i][j] = (T)g.four[i][j];
    for (int a = 0; a < d.n_slip; ++a)
      for (int q = 0; q < 6; ++q) {
        t.sig[a][q] = (T)g.sig[a][q];
        t.sigo[a][q] = (T)(g.sig[a][q] * g.inv_mu);
        t.epso[a][q] = (T)(g.eps[a][q] * g.inv_mu);
      }
    t.c2 = (T)g.c2;
    t.c1nu = (T)g.c1nu;
    // trace-free systems: sigma^a/mu = lam o (eps^a/mu) with lam = (2 C44 x3, C44 x3)
    const double lam[6] = {2 * C44, 2 * C44, 2 * C44, C44, C44, C44};
    double dev = 0.0, scale = 0.0;
    for (int a = 0; a < d.n_slip; ++a)
      for (int q = 0; q < 6; ++q) {
        dev = std::max(dev, std::fabs(g.sig[a][q] - lam[q] * g.eps[a][q]));
        scale = std::max(scale, std::fabs(g.sig[a][q]));
      }
    for (int q = 0; q < 6; ++q) t.lam[q] = (T)lam[q];
    t.tf = dev <= 1e-13 * scale ? 1 : 0;
  };
  fill(g.d);
  fill(g.f);
}

// Core constants with the reference's order of operations.
inline bool build_core(const pfdd_instance_desc &d, Core &c) {
  memset(&c, 0, sizeof c);
  c.flag = d.core_flag;
  const double C44 = d.C44, C12 = d.C12, C11 = d.C11;
  const double mu = C44 - (2.0 * C44 + C12 - C11) / 5.0;
  const double s = mu * d.dslip * d.b;
  switch (d.core_flag) {
    case PFDD_CORE_PERFECT:
    case PFDD_CORE_USFE_ANGLE:
      c.k[0] = d.An / s * M_PI;  // An' pi, core_energy_perfect fft_fftw_slab.cpp:1181,1187
      break;
    case PFDD_CORE_SINE: {
      const double isf = d.isf / s;               // fft_fftw_slab.cpp:1403
      const double Cn = (d.usf - (isf / 2.0)) / s; // fft_fftw_slab.cpp:1405 (uses the scaled isf)
      c.k[0] = isf * M_PI;
      c.k[1] = Cn * 2 * M_PI;
      break;
    }
    case PFDD_CORE_SINE_FIELD:
      c.k[2] = d.isf / s;
      c.k[3] = d.usf / s;
      c.k[4] = 1.0 / (2.0 * s);
      break;
    case PFDD_CORE_MPEA:
      c.k[0] = M_PI / s;   // A(r)/(mu dslip b) pi, fft_fftw_slab.cpp:1231
      break;
    case PFDD_CORE_BCC_PERFECT:
      c.k[0] = d.usf / s * M_PI;   // usf' pi, fft_fftw_slab.cpp:1096,1120
      c.nx = d.nx;
      c.ny = d.ny;
      c.nz = d.nz;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c.four[i][j] = d.four[i][j];
      for (int a = 0; a < d.n_slip; ++a)
        for (int i = 0; i < 3; ++i) {
          c.xn[a][i] = d.xn[a][i];
          c.xb[a][i] = d.xb[a][i];
        }
      break;
    case PFDD_CORE_PYRII:
      for (int n = 1; n <= 4; ++n) {
        c.k[n] = d.aa[n] / s;
        c.k[4 + n] = d.bb[n - 1] / s;
      }
      break;
    case PFDD_CORE_EXTENDED:
      if (d.n_slip % 3) return false;
      c.k[0] = d.c[1] / mu; c.k[1] = d.c[2] / mu; c.k[2] = d.c[3] / mu; c.k[3] = d.c[4] / mu;
      c.k[4] = d.c[5] / mu; c.k[5] = d.c[6] / mu;
      c.k[6] = (2.0 * M_PI) / (d.dslip * d.b);
      c.k[7] = d.c[0] / mu;                  // c0' and 1/(dslip b) of the energy fcore (:1280, :1320)
      c.k[8] = 1.0 / (d.dslip * d.b);
      break;
    default:
      return false;
  }
  // derivatives of f' with respect to the GSFE parameters (adjoint step) and
  // the amplitudes of f itself (energy)
  if (d.core_flag != PFDD_CORE_EXTENDED && d.core_flag != PFDD_CORE_PYRII && d.core_flag != PFDD_CORE_BCC_PERFECT) {
    c.k[7] = M_PI / s;
    c.k[8] = M_PI / (s * s);
    c.k[9] = 2.0 * M_PI / s;
    if (d.core_flag == PFDD_CORE_PERFECT || d.core_flag == PFDD_CORE_USFE_ANGLE) c.k[10] = d.An / s;
    if (d.core_flag == PFDD_CORE_SINE) {
      c.k[10] = d.isf / s;
      c.k[11] = (d.usf - (d.isf / s) / 2.0) / s;
    }
    if (d.core_flag == PFDD_CORE_MPEA) c.k[10] = 1.0 / s;
  }
  if (d.core_flag == PFDD_CORE_BCC_PERFECT) c.k[10] = d.usf / s;   // usf' of the energy density
  for (int i = 0; i < 12; ++i) c.kf[i] = (float)c.k[i];
  return true;
}

inline void build_stress(const pfdd_instance_desc &d, StressArgs &s) {
  memset(&s, 0, sizeof s);
  const double (*p)[3] = d.prim;
  // determinant and inverse as fft.cpp computes them (cofactors / norvol)
  double norvol = p[1][0] * p[2][1] * p[0][2] - p[2][0] * p[1][1] * p[0][2] + p[2][0] * p[0][1] * p[1][2] -
                  p[0][0] * p[2][1] * p[1][2] + p[0][0] * p[1][1] * p[2][2] - p[1][0] * p[0][1] * p[2][2];
  double inv[3][3];
  inv[0][0] = (p[1][1] * p[2][2] - p[2][1] * p[1][2]) / norvol;
  inv[0][1] = (p[2][1] * p[0][2] - p[0][1] * p[2][2]) / norvol;
  inv[0][2] = (p[0][1] * p[1][2] - p[1][1] * p[0][2]) / norvol;
  inv[1][0] = (p[1][2] * p[2][0] - p[2][2] * p[1][0]) / norvol;
  inv[1][1] = (p[2][2] * p[0][0] - p[0][2] * p[2][0]) / norvol;
  inv[1][2] = (p[0][2] * p[1][0] - p[1][2] * p[0][0]) / norvol;
  inv[2][0] = (p[1][0] * p[2][1] - p[2][0] * p[1][1]) / norvol;
  inv[2][1] = (p[2][0] * p[0][1] - p[0][0] * p[2][1]) / norvol;
  inv[2][2] = (p[0][0] * p[1][1] - p[1][0] * p[0][1]) / norvol;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      s.prim[i][j] = p[i][j];
      s.invprim[i][j] = inv[i][j];
      s.dsig[i][j] = d.dsigma[i][j];
    }
  s.ortho = (std::fabs(norvol) < 1.01 && std::fabs(norvol) > 0.99) ? 1 : 0;
  s.S = d.n_slip;
  s.dslip = d.dslip;
  for (int a = 0; a < d.n_slip; ++a)
    for (int i = 0; i < 3; ++i) { s.xn[a][i] = d.xn[a][i]; s.xb[a][i] = d.xb[a][i]; }
  s.ns = d.non_schmid ? 1 : 0;
  if (s.ns) {
    // resolSS_non_Schmid (fft_fftw_slab.cpp:793-828): the maximum resolved
    // shear stress plane at angle_to_110 + 120 a degrees about y, the plane
    // 60 degrees from it, their cross products with b, and the projection
    // S_tot_ij = n_j b_i + w1 n'_j b_i + w2 n_j (n x b)_i + w3 n'_j (n' x b)_i
    double theta = 0.0;
    for (int a = 0; a < d.n_slip && a < 3; ++a) {
      const double n[3] = {-std::sin((theta + d.angle_to_110) * M_PI / 180.), 0.0,
                           std::cos((theta + d.angle_to_110) * M_PI / 180.)};
      const double np[3] = {-std::sin((theta + d.angle_to_110 + 60) * M_PI / 180.), 0.0,
                            std::cos((theta + d.angle_to_110 + 60) * M_PI / 180.)};
      theta += 120.;
      const double *b = d.xb[a];
      const double nb[3] = {n[1] * b[2] - n[2] * b[1], -n[0] * b[2] + n[2] * b[0], n[0] * b[1] - n[1] * b[0]};
      const double npb[3] = {np[1] * b[2] - np[2] * b[1], -np[0] * b[2] + np[2] * b[0], np[0] * b[1] - np[1] * b[0]};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          s.proj[a][i][j] = n[j] * b[i] + d.w1 * np[j] * b[i] + d.w2 * n[j] * nb[i] + d.w3 * np[j] * npb[i];
    }
  }
  s.usfe = d.core_flag == PFDD_CORE_USFE_ANGLE ? 1 : 0;
  const double mu = d.C44 - (2.0 * d.C44 + d.C12 - d.C11) / 5.0;
  s.mu = mu;
  s.s = mu * d.dslip * d.b;
  for (int i = 0; i < 5; ++i) s.fit[i] = d.usfe_fit[i];
  s.fit_sin = std::sin(d.usfe_fit[2] * d.angle_to_110 * M_PI / 180.);
}

// Host twin of the device stress-state step: sigma_rot (rotate_stress,
// fft_fftw_slab.cpp:242-274), tau (resolSS_Schmid / resolSS_non_Schmid) and
// the core model 6 amplitude an[0] = An' pi, an[1] = An' (an may be null).
inline void resolve_state_host(const StressArgs &s, const double (&sigma)[3][3], double *tau, double *an) {
  double sr[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      sr[i][j] = 0.0;
      if (s.ortho) {
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) sr[i][j] += s.prim[i][k] * sigma[k][l] * s.invprim[l][j];
      } else {
        sr[i][j] = sigma[i][j];
      }
    }
  for (int a = 0; a < s.S; ++a) {
    double t = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        t = t + (s.ns ? (sr[i][j] * s.proj[a][i][j]) / s.dslip : (sr[i][j] * s.xn[a][j] * s.xb[a][i]) / s.dslip);
    tau[a] = t;
  }
  if (an) {
    const double ga = s.fit[0] * sr[2][1] * s.mu * 1.0E-9 + s.fit[1];
    const double gc = s.fit[3] * sr[2][1] * s.mu * 1.0E-9 + s.fit[4];
    const double A = ((ga * s.fit_sin + gc) * 1.0E-3) / s.s;
    an[0] = s.usfe ? A * M_PI : 0.0;
    an[1] = s.usfe ? A : 0.0;
  }
}

}  // namespace host
}  // namespace pfdd
