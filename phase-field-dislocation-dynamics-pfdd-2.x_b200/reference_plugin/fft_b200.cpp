/* fft_b200.cpp -- FFT style `b200` (see fft_b200.h). */
#include "fft_b200.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "app.h"
#include "error.h"
#include "material.h"

using namespace PFDD_NS;

FFT_B200::StyleArgs::StyleArgs(int narg, char **arg) : precision(PFDD_FP64), diag_gpu(0), bad(0) {
  for (int i = 0; i < narg; ++i) {
    if (i > 0 && !strcmp(arg[i], "precision") && i + 1 < narg) {
      if (!strcmp(arg[i + 1], "fp32")) precision = PFDD_FP32;
      else if (!strcmp(arg[i + 1], "fp64")) precision = PFDD_FP64;
      else bad = 1;
      ++i;
    } else if (i > 0 && !strcmp(arg[i], "diag") && i + 1 < narg) {
      if (!strcmp(arg[i + 1], "gpu")) diag_gpu = 1;
      else if (!strcmp(arg[i + 1], "host")) diag_gpu = 0;
      else bad = 1;
      ++i;
    } else {
      rest.push_back(arg[i]);
    }
  }
}

FFT_B200::FFT_B200(PFDD_C *p, int narg, char **arg) : FFT_B200(p, StyleArgs(narg, arg)) {}

FFT_B200::FFT_B200(PFDD_C *p, StyleArgs &&a)
    : FFTW_Slab(p, (int)a.rest.size(), a.rest.data()), gpu(nullptr), precision(a.precision), diag_gpu(a.diag_gpu),
      diag_fresh(0) {
  if (a.bad) error->all(FLERR, "Illegal fft_style b200 command: precision fp64|fp32, diag host|gpu");
  // never computed by the reference (src/fft.h:51), read by its exit test
  ximin = 0.0;
}

void FFT_B200::allocate() {
  const int S = app->slip_systems;
  if (app->num_planes < 1 || app->num_planes > S)
    app->num_planes = (app->core_flag == 2 && S >= 3) ? S / 3 : S;
  FFTW_Slab::allocate();
}

FFT_B200::~FFT_B200() {
  if (gpu) pfdd_gpu_destroy(gpu);
}

void FFT_B200::check(int status, const char *what) {
  if (status == PFDD_OK) return;
  char msg[1200];
  snprintf(msg, sizeof msg, "%s: pfdd status %d: %s", what, status, pfdd_gpu_last_error(gpu));
  error->all(FLERR, msg);
}

void FFT_B200::setup() {
  if (diag_gpu) {
    // what the host still reads; the Green's operator lives on the GPU
    rotate_stress();
    frec();
    stiffness();
    // the Voigt constants and eigenstrains Bmatrix also sets (fft_fftw_slab.cpp:483-566)
    const double C44 = material->C44, C12 = material->C12, C11 = material->C11;
    material->mu = C44 - (2.0 * C44 + C12 - C11) / 5.0;
    material->ll = C12 - (2.0 * C44 + C12 - C11) / 5.0;
    material->young = material->mu * (3 * material->ll + 2 * material->mu) / (material->ll + material->mu);
    material->xnu = material->young / 2.0 / material->mu - 1.0;
    for (int i = 0; i < dimension; ++i)
      for (int j = 0; j < dimension; ++j)
        for (int k = 0; k < slip_systems; ++k) eps[k][i][j] = xb[k][i] * xn[k][j] / material->dslip;
  } else {
    FFTW_Slab::setup();
  }
  if (nprocs != 1) error->all(FLERR, "fft_style b200 runs the whole grid on one GPU: use one MPI rank");

  pfdd_instance_desc d;
  memset(&d, 0, sizeof d);
  d.nx = nx; d.ny = ny; d.nz = nz;
  d.n_slip = slip_systems;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      d.four[i][j] = four[i][j];
      d.prim[i][j] = prim[i][j];
      d.sigma[i][j] = sigma[i][j];
      d.dsigma[i][j] = deltasig[i][j];
    }
  for (int a = 0; a < slip_systems; ++a)
    for (int j = 0; j < 3; ++j) {
      d.xn[a][j] = xn[a][j];
      d.xb[a][j] = xb[a][j];
    }
  d.C44 = material->C44; d.C12 = material->C12; d.C11 = material->C11;
  d.dslip = material->dslip; d.b = material->b;
  d.cd_dt = app->CD * app->timestep;
  d.core_flag = app->core_flag;
  d.isf = material->isf; d.usf = material->usf; d.An = material->An;
  const double c[7] = {material->c0, material->c1, material->c2, material->c3, material->c4, material->a1,
                       material->a3};
  for (int i = 0; i < 7; ++i) d.c[i] = c[i];
  const double aa[5] = {material->aa0, material->aa1, material->aa2, material->aa3, material->aa4};
  for (int i = 0; i < 5; ++i) d.aa[i] = aa[i];
  const double bb[4] = {material->bb1, material->bb2, material->bb3, material->bb4};
  for (int i = 0; i < 4; ++i) d.bb[i] = bb[i];
  d.site_gsfe = app->core_flag == PFDD_CORE_MPEA ? material->A_mpea : nullptr;
  const size_t n = (size_t)slip_systems * nx * ny * nz;
  bool masked = false;
  for (size_t i = 0; i < n && !masked; ++i) masked = xo[i] != 0.0;
  d.xo = masked ? xo : nullptr;
  d.non_schmid = app->non_Schmid;
  d.angle_to_110 = app->angle_to_110;
  d.w1 = app->w1; d.w2 = app->w2; d.w3 = app->w3;
  const double fit[5] = {material->a_slope, material->a_b, material->b_b, material->c_slope, material->c_b};
  for (int i = 0; i < 5; ++i) d.usfe_fit[i] = fit[i];

  pfdd_options o;
  memset(&o, 0, sizeof o);
  o.precision = precision;
  o.imag_mode = PFDD_IMAG_AUTO;
  o.device = 0;
  o.use_graphs = 1;
  o.check_finite = 1;
  if (gpu) pfdd_gpu_destroy(gpu);
  gpu = nullptr;
  check(pfdd_gpu_create(&d, 1, &o, &gpu), "pfdd_gpu_create");
  // The first GL iteration of the reference reads data_fftw (core force and
  // transform) and updates xi; every initial_sxtal_* used by the decks sets
  // them equal.  The GPU steps one state, xi.
  for (size_t i = 0; i < n; ++i)
    if (data_fftw[i].re != xi[0][2 * i] || data_fftw[i].im != xi[0][2 * i + 1]) {
      if (me == 0) printf("fft_style b200: data_fftw differs from xi after the initial condition; the GPU starts from xi\n");
      break;
    }
  push_xi();
}

void FFT_B200::push_xi() { check(pfdd_gpu_set_state_interleaved(gpu, 0, xi[0]), "pfdd_gpu_set_state_interleaved"); }

void FFT_B200::pull_xi() { check(pfdd_gpu_get_state_interleaved(gpu, 0, xi[0]), "pfdd_gpu_get_state_interleaved"); }

void FFT_B200::set_device_stress() {
  double s[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s[i][j] = sigma[i][j];
  check(pfdd_gpu_set_stress(gpu, 0, s), "pfdd_gpu_set_stress");
}

pfdd_step_stats FFT_B200::advance(int n, double tol) {
  pfdd_step_stats st;
  memset(&st, 0, sizeof st);
  // one stress state of up to n iterations; the host keeps sigma (the device
  // adds deltasig when its state ends, so this state's sigma goes first)
  set_device_stress();
  check(pfdd_gpu_advance(gpu, n, 1, tol, &st), "pfdd_gpu_advance");
  xinorm = st.xinorm;
  xiave = st.xiave;
  diag_fresh = 0;
  return st;
}

// ---- strain / stress from the GPU (diag gpu) ------------------------------
void FFT_B200::gpu_diagnostics() {
  const size_t N = (size_t)nx * ny * nz;
  std::vector<double> e(9 * N), s(9 * N);
  double ae[9], as[9];
  check(pfdd_gpu_strain_stress(gpu, 0, e.data(), s.data(), ae, as), "pfdd_gpu_strain_stress");
  // data_eps / data_sigma: 2*(r + ida*N + idb*3N) (fft_fftw_slab.cpp:3355, 3520)
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const double *pe = e.data() + (3 * a + b) * N, *ps = s.data() + (3 * a + b) * N;
      for (size_t r = 0; r < N; ++r) {
        const size_t na = 2 * (r + a * N + b * 3 * N);
        data_eps[na] = pe[r];
        data_eps[na + 1] = 0.0;
        data_sigma[na] = ps[r];
        data_sigma[na + 1] = 0.0;
      }
      ave_eps[a][b] = ae[3 * a + b];
      ave_sigma[a][b] = as[3 * a + b];
    }
  diag_fresh = 1;
}

void FFT_B200::strain() {
  if (!diag_gpu) { FFTW_Slab::strain(); return; }
  gpu_diagnostics();
}

void FFT_B200::total_average_strain() {
  if (!diag_gpu) FFTW_Slab::total_average_strain();
}

void FFT_B200::stress() {
  if (!diag_gpu) { FFTW_Slab::stress(); return; }
  if (!diag_fresh) gpu_diagnostics();
}
