// FP64 3-D FFT behind the FFTW 2.1.5 MPI API (declarations in dfftw_mpi.h).
// Test infrastructure only: it lets the reference PFDD sources build into a
// CPU oracle in a container without FFTW.
//
// Algorithm: self-sorting (Stockham) mixed-radix decimation in frequency.
// A length-n transform with first radix p, m = n/p, stride s maps
//   y[q + s*(p*j + k)] = w_n^(j*k) * sum_r x[q + s*(j + r*m)] * w_p^(r*k)
// and recurses on length m with stride s*p, ping-ponging between two
// buffers.  Every element is itself a contiguous "vector" of V complex values,
// so the y- and x-axis passes stream whole rows/planes (V = nz or ny*nz, times
// the number of interleaved fields) and the z-axis pass loops over lines.
// Radices 4, 2, 3, 5 are written out; any other prime factor uses a direct
// O(p^2) DFT.  Twiddles are cos/sin of 2*pi*(j*k mod n)/n in double.
#include "dfftw_mpi.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <map>
#include <thread>
#include <utility>
#include <vector>

namespace {

struct Stage {
  int p;                 // radix
  int m;                 // n / (product of radices up to and including this one)
  int s;                 // stride on entry
  std::vector<double> tw;  // (m * p) complex twiddles w_n^(j*k), laid out [j][k]
};

struct Plan1D {
  int n;
  int sign;
  std::vector<Stage> stages;
};

std::map<std::pair<int, int>, Plan1D *> g_plans;
double g_flops = 0.0;

Plan1D *get_plan(int n, int sign) {
  auto key = std::make_pair(n, sign);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) return it->second;
  Plan1D *pl = new Plan1D;
  pl->n = n;
  pl->sign = sign;
  int rem = n, s = 1, len = n;
  while (rem > 1) {
    int p;
    if (rem % 4 == 0) p = 4;
    else if (rem % 2 == 0) p = 2;
    else if (rem % 3 == 0) p = 3;
    else if (rem % 5 == 0) p = 5;
    else {
      p = 7;
      while (rem % p) p += 2;
    }
    Stage st;
    st.p = p;
    st.m = len / p;
    st.s = s;
    st.tw.resize(2 * (size_t)st.m * p);
    for (int j = 0; j < st.m; ++j)
      for (int k = 0; k < p; ++k) {
        long long e = ((long long)j * k) % len;
        double ang = 2.0 * M_PI * (double)e / (double)len;
        st.tw[2 * ((size_t)j * p + k)] = std::cos(ang);
        st.tw[2 * ((size_t)j * p + k) + 1] = sign * std::sin(ang);
      }
    pl->stages.push_back(st);
    rem /= p;
    s *= p;
    len /= p;
  }
  g_plans[key] = pl;
  return pl;
}

// One Stockham stage on V-vectors: x -> y, vector components [v0, v1) only
// (components are independent, so disjoint ranges can run on separate threads).
void run_stage(const Stage &st, int sign, const double *x, double *y, int V, int v0, int v1) {
  const int p = st.p, m = st.m, s = st.s;
  const size_t sv = (size_t)s * V;  // doubles per "q-run" is 2*sv
  const double c3 = -0.5, s3 = sign * std::sqrt(3.0) * 0.5;
  const double c51 = std::cos(2 * M_PI / 5), c52 = std::cos(4 * M_PI / 5);
  const double s51 = sign * std::sin(2 * M_PI / 5), s52 = sign * std::sin(4 * M_PI / 5);
  std::vector<double> ar, ai;
  if (p > 5) { ar.resize(p); ai.resize(p); }
  for (int j = 0; j < m; ++j) {
    const double *tw = &st.tw[2 * (size_t)j * p];
    for (size_t q0 = 0; q0 < sv; q0 += V)
    for (size_t qv = q0 + v0; qv < q0 + v1; ++qv) {
      // input r: index (j + r*m) * s  (+q) ; vector offset folded into qv
      const double *in0 = x + 2 * ((size_t)j * sv + qv);
      const size_t istep = 2 * (size_t)m * sv;
      double *out0 = y + 2 * ((size_t)p * j * sv + qv);
      const size_t ostep = 2 * sv;
      if (p == 2) {
        double a0r = in0[0], a0i = in0[1], a1r = in0[istep], a1i = in0[istep + 1];
        double b1r = a0r - a1r, b1i = a0i - a1i;
        out0[0] = a0r + a1r; out0[1] = a0i + a1i;
        out0[ostep] = b1r * tw[2] - b1i * tw[3];
        out0[ostep + 1] = b1r * tw[3] + b1i * tw[2];
      } else if (p == 4) {
        double a0r = in0[0], a0i = in0[1];
        double a1r = in0[istep], a1i = in0[istep + 1];
        double a2r = in0[2 * istep], a2i = in0[2 * istep + 1];
        double a3r = in0[3 * istep], a3i = in0[3 * istep + 1];
        double t0r = a0r + a2r, t0i = a0i + a2i, t1r = a0r - a2r, t1i = a0i - a2i;
        double t2r = a1r + a3r, t2i = a1i + a3i, t3r = a1r - a3r, t3i = a1i - a3i;
        // multiply t3 by sign*i : (sign*i)*(t3r + i t3i) = -sign*t3i + i sign*t3r
        double u3r = -sign * t3i, u3i = sign * t3r;
        double b0r = t0r + t2r, b0i = t0i + t2i;
        double b2r = t0r - t2r, b2i = t0i - t2i;
        double b1r = t1r + u3r, b1i = t1i + u3i;
        double b3r = t1r - u3r, b3i = t1i - u3i;
        out0[0] = b0r; out0[1] = b0i;
        out0[ostep] = b1r * tw[2] - b1i * tw[3];
        out0[ostep + 1] = b1r * tw[3] + b1i * tw[2];
        out0[2 * ostep] = b2r * tw[4] - b2i * tw[5];
        out0[2 * ostep + 1] = b2r * tw[5] + b2i * tw[4];
        out0[3 * ostep] = b3r * tw[6] - b3i * tw[7];
        out0[3 * ostep + 1] = b3r * tw[7] + b3i * tw[6];
      } else if (p == 3) {
        double a0r = in0[0], a0i = in0[1];
        double a1r = in0[istep], a1i = in0[istep + 1];
        double a2r = in0[2 * istep], a2i = in0[2 * istep + 1];
        double sr = a1r + a2r, si = a1i + a2i, dr = a1r - a2r, di = a1i - a2i;
        double b0r = a0r + sr, b0i = a0i + si;
        double mr = a0r + c3 * sr, mi = a0i + c3 * si;
        // w3 = c3 + i*s3 ; b1 = a0 + w a1 + w^2 a2 = m + i s3 d
        double b1r = mr - s3 * di, b1i = mi + s3 * dr;
        double b2r = mr + s3 * di, b2i = mi - s3 * dr;
        out0[0] = b0r; out0[1] = b0i;
        out0[ostep] = b1r * tw[2] - b1i * tw[3];
        out0[ostep + 1] = b1r * tw[3] + b1i * tw[2];
        out0[2 * ostep] = b2r * tw[4] - b2i * tw[5];
        out0[2 * ostep + 1] = b2r * tw[5] + b2i * tw[4];
      } else if (p == 5) {
        double a0r = in0[0], a0i = in0[1];
        double a1r = in0[istep], a1i = in0[istep + 1];
        double a2r = in0[2 * istep], a2i = in0[2 * istep + 1];
        double a3r = in0[3 * istep], a3i = in0[3 * istep + 1];
        double a4r = in0[4 * istep], a4i = in0[4 * istep + 1];
        double s14r = a1r + a4r, s14i = a1i + a4i, d14r = a1r - a4r, d14i = a1i - a4i;
        double s23r = a2r + a3r, s23i = a2i + a3i, d23r = a2r - a3r, d23i = a2i - a3i;
        double b0r = a0r + s14r + s23r, b0i = a0i + s14i + s23i;
        double m1r = a0r + c51 * s14r + c52 * s23r, m1i = a0i + c51 * s14i + c52 * s23i;
        double m2r = a0r + c52 * s14r + c51 * s23r, m2i = a0i + c52 * s14i + c51 * s23i;
        double n1r = s51 * d14r + s52 * d23r, n1i = s51 * d14i + s52 * d23i;
        double n2r = s52 * d14r - s51 * d23r, n2i = s52 * d14i - s51 * d23i;
        double b[10] = {b0r, b0i, m1r - n1i, m1i + n1r, m2r - n2i, m2i + n2r,
                        m2r + n2i, m2i - n2r, m1r + n1i, m1i - n1r};
        out0[0] = b[0]; out0[1] = b[1];
        for (int k = 1; k < 5; ++k) {
          double br = b[2 * k], bi = b[2 * k + 1];
          out0[k * ostep] = br * tw[2 * k] - bi * tw[2 * k + 1];
          out0[k * ostep + 1] = br * tw[2 * k + 1] + bi * tw[2 * k];
        }
      } else {
        for (int r = 0; r < p; ++r) { ar[r] = in0[r * istep]; ai[r] = in0[r * istep + 1]; }
        for (int k = 0; k < p; ++k) {
          double br = 0, bi = 0;
          for (int r = 0; r < p; ++r) {
            long long e = ((long long)r * k) % p;
            double c = std::cos(2 * M_PI * e / p), sn = sign * std::sin(2 * M_PI * e / p);
            br += ar[r] * c - ai[r] * sn;
            bi += ar[r] * sn + ai[r] * c;
          }
          out0[k * ostep] = br * tw[2 * k] - bi * tw[2 * k + 1];
          out0[k * ostep + 1] = br * tw[2 * k + 1] + bi * tw[2 * k];
        }
      }
    }
  }
}

// Worker threads of one transform: PFDD_SHIM_THREADS (default 1).  The
// reference's FFTW-MPI build spreads its transforms over the MPI ranks; this
// single-rank stand-in spreads them over threads instead.  Every element is
// computed by the same operations in the same order whatever the count, so
// the results are bit-identical.
int shim_threads() {
  static int t = -1;
  if (t < 0) {
    const char *e = getenv("PFDD_SHIM_THREADS");
    t = e ? std::max(1, atoi(e)) : 1;
  }
  return t;
}

template <class F>
void parallel_for(int count, F body) {
  const int T = std::min(shim_threads(), count);
  if (T <= 1) {
    body(0, count, 0);
    return;
  }
  std::vector<std::thread> th;
  for (int k = 0; k < T; ++k) {
    const int a = (int)((long long)count * k / T), b = (int)((long long)count * (k + 1) / T);
    th.emplace_back([=] { body(a, b, k); });
  }
  for (auto &x : th) x.join();
}

// `count` independent transforms of length n whose elements are V-vectors:
// element (t, i, v) at data[(t*n + i)*V + v]; scratch holds count*n*V complex.
// Threads take whole transforms when there are several, else ranges of v.
void fft_lines(double *data, double *scratch, int count, int n, int V, int sign) {
  if (n <= 1) return;
  Plan1D *pl = get_plan(n, sign);
  const size_t tsz = 2 * (size_t)n * V;
  auto one = [&](int t, int v0, int v1) {
    double *a = data + t * tsz, *b = scratch + t * tsz;
    for (const Stage &st : pl->stages) {
      run_stage(st, sign, a, b, V, v0, v1);
      std::swap(a, b);
    }
    if (a != data + t * tsz)
      for (int i = 0; i < n; ++i)
        std::memcpy(data + t * tsz + 2 * ((size_t)i * V + v0), a + 2 * ((size_t)i * V + v0),
                    2 * (size_t)(v1 - v0) * sizeof(double));
  };
  if (count >= shim_threads())
    parallel_for(count, [&](int t0, int t1, int) {
      for (int t = t0; t < t1; ++t) one(t, 0, V);
    });
  else
    for (int t = 0; t < count; ++t)
      parallel_for(V, [&](int v0, int v1, int) { one(t, v0, v1); });
  g_flops += 5.0 * n * std::log2((double)n) * (double)count * V;
}

}  // namespace

struct pfdd_shim_plan3d {
  int nx, ny, nz, sign;
};

fftwnd_mpi_plan fftw3d_mpi_create_plan(MPI_Comm, int nx, int ny, int nz,
                                       fftw_direction dir, int) {
  fftwnd_mpi_plan p = new pfdd_shim_plan3d;
  p->nx = nx; p->ny = ny; p->nz = nz;
  p->sign = (dir == FFTW_FORWARD) ? -1 : 1;
  return p;
}

void fftwnd_mpi_local_sizes(fftwnd_mpi_plan p, int *local_nx, int *local_x_start,
                            int *local_ny_after_transpose,
                            int *local_y_start_after_transpose,
                            int *total_local_size) {
  *local_nx = p->nx;
  *local_x_start = 0;
  *local_ny_after_transpose = p->ny;
  *local_y_start_after_transpose = 0;
  *total_local_size = p->nx * p->ny * p->nz;
}

void fftwnd_mpi(fftwnd_mpi_plan p, int n_fields, fftw_complex *local_data,
                fftw_complex *, fftwnd_mpi_output_order) {
  const int nx = p->nx, ny = p->ny, nz = p->nz, h = n_fields;
  double *d = reinterpret_cast<double *>(local_data);
  size_t total = (size_t)nx * ny * nz * h;
  std::vector<double> scratch(2 * total);
  // z: lines of nz elements (vector = fields).  Lines are gathered in groups
  // of B into a [nz][B*h] block so the butterfly loops run over contiguous
  // vectors, then scattered back.
  const int lines = nx * ny;
  const int B = 8;
  const int groups = (lines + B - 1) / B;
  Plan1D *pl = nz > 1 ? get_plan(nz, p->sign) : nullptr;   // plans are built outside the threads
  parallel_for(groups, [&](int g0, int g1, int) {
    std::vector<double> blk(2 * (size_t)nz * B * h), bsc(2 * (size_t)nz * B * h);
    for (int l0 = g0 * B; l0 < std::min(lines, g1 * B); l0 += B) {
      const int nb = std::min(B, lines - l0);
      const int V = nb * h;
      for (int b = 0; b < nb; ++b)
        for (int i = 0; i < nz; ++i)
          for (int f = 0; f < h; ++f) {
            const double *src = d + 2 * (((size_t)(l0 + b) * nz + i) * h + f);
            double *dst = blk.data() + 2 * ((size_t)i * V + b * h + f);
            dst[0] = src[0]; dst[1] = src[1];
          }
      if (nz > 1) {
        double *a = blk.data(), *c = bsc.data();
        for (const Stage &st : pl->stages) {
          run_stage(st, p->sign, a, c, V, 0, V);
          std::swap(a, c);
        }
        if (a != blk.data()) std::memcpy(blk.data(), a, 2 * (size_t)nz * V * sizeof(double));
      }
      for (int b = 0; b < nb; ++b)
        for (int i = 0; i < nz; ++i)
          for (int f = 0; f < h; ++f) {
            double *dst = d + 2 * (((size_t)(l0 + b) * nz + i) * h + f);
            const double *src = blk.data() + 2 * ((size_t)i * V + b * h + f);
            dst[0] = src[0]; dst[1] = src[1];
          }
    }
  });
  if (nz > 1) g_flops += 5.0 * nz * std::log2((double)nz) * (double)lines * h;
  // y: nx transforms of ny elements, vector = nz*fields
  fft_lines(d, scratch.data(), nx, ny, nz * h, p->sign);
  // x: one transform of nx elements, vector = ny*nz*fields
  fft_lines(d, scratch.data(), 1, nx, ny * nz * h, p->sign);
}

void fftwnd_mpi_destroy_plan(fftwnd_mpi_plan p) { delete p; }

extern "C" double pfdd_shim_fft_flops(void) { return g_flops; }

// Plain-C entry for the shim self-test: in-place 3-D transform of an
// interleaved complex array [nx][ny][nz][h].
extern "C" void pfdd_shim_fft3d(double *data, int nx, int ny, int nz, int h, int sign) {
  pfdd_shim_plan3d p{nx, ny, nz, sign < 0 ? -1 : 1};
  fftwnd_mpi(&p, h, reinterpret_cast<fftw_complex *>(data), nullptr, FFTW_NORMAL_ORDER);
}
