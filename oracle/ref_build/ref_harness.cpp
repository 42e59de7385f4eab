// Oracle harness: drives the reference PFDD sources (compiled unmodified with
// the single-rank MPI and FFTW-2 stand-ins in this directory) through one
// deck, with hooks a test needs.  Test infrastructure only.
//
//   pfdd_ref_harness -deck in.deck [-steps N] [-state_in xi0.bin] [-xo_in xo.bin]
//       [-mpea_in a.bin] [-set key value]... [-state_out xi.bin] [-stats_out s.txt]
//       [-setup_out setup.txt] [-B_out bb.bin] [-stress_out st.bin] [-profile_out pr.bin] [-timing]
//       [-cond_steps n -cond_out cond.bin [-cond_in c0.bin]]
//
// Sequence (mirrors App::run, app.cpp:127-205, with the `run` command taken
// out of the deck so state can be injected between init and setup):
//   deck lines (except `run`) -> input->one()
//   app->stoptime = time + T;  app->init()      (fft->init, set_slip, initial_sxtal)
//   [inject]  xi, data_fftw, xo, material scalars, per-site GSFE amplitude
//   timer->init(); app->setup(); app->iterate()  (SolveGL::iterate)
//   [dump]    xi[0] (2*S*N doubles, reference layout), per-step xinorm/xiave
//   [stress]  the strain/stress diagnostics of the final state as DiagStress
//             computes them (diag_stress.cpp:43-62: averages reset, strain,
//             total_average_strain, stress), after prep_forward() so data_fftw
//             holds the transform of that state: data_eps (2*9*N), data_sigma
//             (2*9*N), ave_eps[3][3], ave_sigma[3][3], avepst[3][3]
//
// Injection targets are the reference's own public members: FFT::xi/xo
// (fft.h:48-50), FFTW_Slab::data_fftw (fft_fftw_slab.h), Material scalars
// (material.h).  Uninitialised reference members that change control flow are
// set explicitly: FFT::ximin (fft.h:51, read at solve_GL.cpp:108,142) = 0 and
// App::num_planes (app.h) = S, or S/3 for core_energy 2.
#include <sys/mman.h>
#include <sys/wait.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mpi.h"
#include "PFDD.h"
#include "app.h"
#include "fft.h"
#include "input.h"
#include "material.h"
#include "memory.h"
#include "timer.h"
#include "solve.h"
#include "oracle_slab.h"

using namespace PFDD_NS;

void OracleSlab::allocate() {
  FFTW_Slab::allocate();
  int n = local_x * local_y * local_z;
  int nmax = slip_systems > num_planes ? slip_systems : num_planes;
  memory->destroy(gradx); memory->create(gradx, nmax * n, "gradx");
  memory->destroy(grady); memory->create(grady, nmax * n, "grady");
  memory->destroy(gradz); memory->create(gradz, nmax * n, "gradz");
  memory->destroy(theta); memory->create(theta, nmax * n, "theta");
  memory->destroy(fcore); memory->create(fcore, nmax * n, "fcore");
  memory->destroy(f_core); memory->create(f_core, nmax * n, "f_core");
  for (int i = 0; i < nmax * n; ++i) gradx[i] = grady[i] = gradz[i] = theta[i] = 0.0;
}

void OracleSlab::update_order_parameter() {
  FFTW_Slab::update_order_parameter();
  step_xinorm.push_back(xinorm);
  step_xiave.push_back(xiave);
}

static int setup_procs() {
  const char *e = getenv("PFDD_ORACLE_SETUP_PROCS");
  return e ? atoi(e) : 1;
}

// Bmatrix / Fmatrix on forked one-x-plane slabs (see oracle_slab.h).  Each
// table is [comps][local_x*ny*nz] (BB: ka + kb*S; FF, DD: ka + i*S + j*3S);
// a slab call lays out its plane as [comps][ny*nz], copied into place here.
void OracleSlab::slab_call(int which) {
  if (which == 0) FFTW_Slab::Bmatrix();
  else FFTW_Slab::Fmatrix();
}

void OracleSlab::forked_setup(int which, SlabOut *outs, int nouts) {
  const int lx = local_x, lx0 = local_x_start;
  const size_t plane = (size_t)local_y * local_z, n = (size_t)lx * plane;
  int P = setup_procs();
  if (P > lx) P = lx;
  // the scalars and small tables the call also sets (material mu/ll/young/xnu,
  // eps): one plane in this process, into scratch
  std::vector<std::vector<double>> scratch(nouts);
  std::vector<double *> saved(nouts);
  for (int o = 0; o < nouts; ++o) {
    saved[o] = *outs[o].member;
    scratch[o].resize((size_t)outs[o].comps * plane);
    *outs[o].member = scratch[o].data();
  }
  local_x = 1;
  slab_call(which);
  local_x = lx;
  // shared mappings replace the tables (the reference never frees them)
  std::vector<double *> shared(nouts);
  for (int o = 0; o < nouts; ++o) {
    size_t bytes = (size_t)outs[o].comps * n * sizeof(double);
    void *m = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (m == MAP_FAILED) { fprintf(stderr, "harness: mmap of %zu bytes failed\n", bytes); exit(2); }
    shared[o] = static_cast<double *>(m);
    if (saved[o]) memory->destroy(saved[o]);
  }
  std::vector<pid_t> kids;
  for (int r = 0; r < P; ++r) {
    pid_t pid = fork();
    if (pid < 0) { fprintf(stderr, "harness: fork failed\n"); exit(2); }
    if (pid == 0) {
      if (!freopen("/dev/null", "w", stdout)) _exit(3);   // the set-up's per-call prints
      for (int x = r; x < lx; x += P) {
        local_x = 1;
        local_x_start = lx0 + x;
        frec();
        for (int o = 0; o < nouts; ++o) *outs[o].member = scratch[o].data();
        slab_call(which);
        for (int o = 0; o < nouts; ++o)
          for (int c = 0; c < outs[o].comps; ++c)
            memcpy(shared[o] + (size_t)c * n + (size_t)x * plane, scratch[o].data() + (size_t)c * plane,
                   plane * sizeof(double));
      }
      _exit(0);
    }
    kids.push_back(pid);
  }
  for (pid_t k : kids) {
    int status = 0;
    if (waitpid(k, &status, 0) < 0 || !WIFEXITED(status) || WEXITSTATUS(status) != 0) {
      fprintf(stderr, "harness: a set-up process failed\n");
      exit(2);
    }
  }
  local_x = lx;
  local_x_start = lx0;
  for (int o = 0; o < nouts; ++o) *outs[o].member = shared[o];
}

void OracleSlab::Bmatrix() {
  if (setup_procs() <= 1 || local_x < 2) { FFTW_Slab::Bmatrix(); return; }
  SlabOut o[1] = {{&BB, slip_systems * slip_systems}};
  forked_setup(0, o, 1);
}

void OracleSlab::Fmatrix() {
  if (setup_procs() <= 1 || local_x < 2) { FFTW_Slab::Fmatrix(); return; }
  SlabOut o[2] = {{&FF, 9 * slip_systems}, {&DD, 9 * slip_systems}};
  forked_setup(1, o, 2);
}

#ifndef PFDD_ORACLE_SLAB_ONLY
static std::vector<double> read_bin(const char *path, size_t expect) {
  FILE *f = fopen(path, "rb");
  if (!f) { fprintf(stderr, "harness: cannot open %s\n", path); exit(2); }
  std::vector<double> v(expect);
  size_t got = fread(v.data(), sizeof(double), expect, f);
  fclose(f);
  if (got != expect) {
    fprintf(stderr, "harness: %s holds %zu doubles, expected %zu\n", path, got, expect);
    exit(2);
  }
  return v;
}

static void write_bin(const char *path, const double *p, size_t n) {
  FILE *f = fopen(path, "wb");
  if (!f) { fprintf(stderr, "harness: cannot write %s\n", path); exit(2); }
  fwrite(p, sizeof(double), n, f);
  fclose(f);
}

static double *material_field(Material *m, const std::string &k) {
  if (k == "b") return &m->b;
  if (k == "mu") return &m->mu;
  if (k == "young") return &m->young;
  if (k == "isf") return &m->isf;
  if (k == "usf") return &m->usf;
  if (k == "An") return &m->An;
  if (k == "Cn") return &m->Cn;
  if (k == "c0") return &m->c0;
  if (k == "c1") return &m->c1;
  if (k == "c2") return &m->c2;
  if (k == "c3") return &m->c3;
  if (k == "c4") return &m->c4;
  if (k == "a1") return &m->a1;
  if (k == "a3") return &m->a3;
  if (k == "aa0") return &m->aa0;
  if (k == "aa1") return &m->aa1;
  if (k == "aa2") return &m->aa2;
  if (k == "aa3") return &m->aa3;
  if (k == "aa4") return &m->aa4;
  if (k == "bb1") return &m->bb1;
  if (k == "bb2") return &m->bb2;
  if (k == "bb3") return &m->bb3;
  if (k == "bb4") return &m->bb4;
  if (k == "dslip") return &m->dslip;
  return nullptr;
}

int main(int argc, char **argv) {
  const char *deck = nullptr, *state_in = nullptr, *xo_in = nullptr, *mpea_in = nullptr;
  const char *state_out = nullptr, *stats_out = nullptr, *setup_out = nullptr, *B_out = nullptr,
             *stress_out = nullptr, *profile_out = nullptr, *cond_out = nullptr, *cond_in = nullptr;
  long cond_steps = 0;
  long steps_override = -1;
  bool timing = false;
  std::vector<std::pair<std::string, double>> sets;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto need = [&](int k) {
      if (i + k >= argc) { fprintf(stderr, "harness: %s needs %d value(s)\n", a.c_str(), k); exit(2); }
    };
    if (a == "-deck") { need(1); deck = argv[++i]; }
    else if (a == "-steps") { need(1); steps_override = atol(argv[++i]); }
    else if (a == "-state_in") { need(1); state_in = argv[++i]; }
    else if (a == "-xo_in") { need(1); xo_in = argv[++i]; }
    else if (a == "-mpea_in") { need(1); mpea_in = argv[++i]; }
    else if (a == "-state_out") { need(1); state_out = argv[++i]; }
    else if (a == "-stats_out") { need(1); stats_out = argv[++i]; }
    else if (a == "-setup_out") { need(1); setup_out = argv[++i]; }
    else if (a == "-B_out") { need(1); B_out = argv[++i]; }
    else if (a == "-stress_out") { need(1); stress_out = argv[++i]; }
    else if (a == "-profile_out") { need(1); profile_out = argv[++i]; }
    else if (a == "-cond_steps") { need(1); cond_steps = atol(argv[++i]); }
    else if (a == "-cond_out") { need(1); cond_out = argv[++i]; }
    else if (a == "-cond_in") { need(1); cond_in = argv[++i]; }
    else if (a == "-set") { need(2); sets.emplace_back(argv[i + 1], atof(argv[i + 2])); i += 2; }
    else if (a == "-timing") { timing = true; }
    else { fprintf(stderr, "harness: unknown option %s\n", a.c_str()); return 2; }
  }
  if (!deck) { fprintf(stderr, "harness: -deck is required\n"); return 2; }

  MPI_Init(&argc, &argv);
  char a0[] = "pfdd", a1[] = "-log", a2[] = "none", a3[] = "-screen", a4[] = "none";
  char *pargv[] = {a0, a1, a2, a3, a4, nullptr};
  PFDD_C *pfdd = new PFDD_C(5, pargv, MPI_COMM_WORLD);

  FILE *fd = fopen(deck, "r");
  if (!fd) { fprintf(stderr, "harness: cannot open deck %s\n", deck); return 2; }
  char line[4096];
  double run_T = 1.0;
  bool saw_run = false;
  while (fgets(line, sizeof line, fd)) {
    char word[256] = {0}, second[256] = {0};
    if (sscanf(line, "%255s %255s", word, second) < 1 || word[0] == '#') continue;
    if (strcmp(word, "run") == 0) { run_T = atof(second); saw_run = true; continue; }
    std::string l = line;
    if (strcmp(word, "fft_style") == 0 && strcmp(second, "fftw_slab") == 0) {
      size_t p = l.find("fftw_slab");
      l.replace(p, 9, "fftw_slab_oracle");
    }
    pfdd->input->one(l.c_str());
    if (strcmp(word, "app_style") == 0) {
      App *app = pfdd->app;
      app->num_planes = (app->core_flag == 2) ? app->slip_systems / 3 : app->slip_systems;
      if (app->num_planes < 1) app->num_planes = 1;
    }
  }
  fclose(fd);
  if (!saw_run) { fprintf(stderr, "harness: deck has no run command\n"); return 2; }

  App *app = pfdd->app;
  OracleSlab *fft = dynamic_cast<OracleSlab *>(pfdd->fft);
  if (!fft) { fprintf(stderr, "harness: deck must use fft_style fftw_slab\n"); return 2; }

  app->stoptime = app->time + run_T;
  app->stopsteps = -1;
  app->init();
  fft->ximin = 0.0;

  const int S = fft->slip_systems;
  const size_t N = (size_t)fft->nx * fft->ny * fft->nz;
  Material *mat = fft->material;
  for (auto &kv : sets) {
    double *f = material_field(mat, kv.first);
    if (kv.first == "CD") { app->CD = kv.second; continue; }
    if (kv.first == "timestep") { app->timestep = kv.second; continue; }
    if (!f) { fprintf(stderr, "harness: unknown -set key %s\n", kv.first.c_str()); return 2; }
    *f = kv.second;
  }
  if (state_in) {
    std::vector<double> xi = read_bin(state_in, 2 * (size_t)S * N);
    for (size_t i = 0; i < (size_t)S * N; ++i) {
      fft->xi[0][2 * i] = xi[2 * i];
      fft->xi[0][2 * i + 1] = xi[2 * i + 1];
      fft->data_fftw[i].re = xi[2 * i];
      fft->data_fftw[i].im = xi[2 * i + 1];
    }
  } else {
    // initial_sxtal_* leaves data_fftw unset away from the seeded sites
    // (e.g. fft_fftw_slab.cpp:2905-2922); make the first step read xi.
    for (size_t i = 0; i < (size_t)S * N; ++i) {
      fft->data_fftw[i].re = fft->xi[0][2 * i];
      fft->data_fftw[i].im = fft->xi[0][2 * i + 1];
    }
  }
  if (xo_in) {
    std::vector<double> xo = read_bin(xo_in, (size_t)S * N);
    for (size_t i = 0; i < (size_t)S * N; ++i) fft->xo[i] = xo[i];
  }
  if (mpea_in) {
    std::vector<double> am = read_bin(mpea_in, (size_t)S * N);
    mat->A_mpea = new double[(size_t)S * N];
    for (size_t i = 0; i < (size_t)S * N; ++i) mat->A_mpea[i] = am[i];
  }
  if (steps_override >= 0) {
    // steps = stress states * GL iterations; keep one stress state.
    app->stopsteps = 1;
    pfdd->solve->max_iter = (int)steps_override;
  }

  pfdd->timer->init();
  app->setup();
  if (cond_steps > 0) {
    // The conductivity sub-problem alone, in SolveGLCond's order
    // (solve_GL+cond.cpp:96-122): it reads none of the dislocation fields.
    // condxi's imaginary half and conddata_fftw are never initialised by the
    // reference (fft_fftw_slab.cpp:146, :170-173): start both from cond_in or 0.
    std::vector<double> c0 = cond_in ? read_bin(cond_in, 2 * N) : std::vector<double>(2 * N, 0.0);
    for (size_t i = 0; i < N; ++i) {
      fft->condxi[0][2 * i] = c0[2 * i];
      fft->condxi[0][2 * i + 1] = c0[2 * i + 1];
      fft->conddata_fftw[i].re = c0[2 * i];
      fft->conddata_fftw[i].im = c0[2 * i + 1];
    }
    std::vector<double> rec, fields;
    for (long it = 0; it < cond_steps; ++it) {
      fft->forwardcond();
      fft->divcurrent();
      fft->backwardcond();
      rec.push_back(fft->conductivity);
      if (it == 0) {
        // the parts of the first iteration the reference defines: the
        // unnormalised inverse transforms a (jcurrent_fftw), b (conddata_bpart)
        // and j (jcurrent).  Its conddata_real also reads condsigma_array[j+1]
        // before writing it (fft_fftw_slab.cpp:2108 vs :2176-2181).
        for (size_t i = 0; i < N; ++i) {
          fields.push_back(fft->jcurrent_fftw[i].re); fields.push_back(fft->jcurrent_fftw[i].im);
        }
        for (size_t i = 0; i < N; ++i) {
          fields.push_back(fft->conddata_bpart[i].re); fields.push_back(fft->conddata_bpart[i].im);
        }
        for (size_t i = 0; i < N; ++i) {
          fields.push_back(fft->jcurrent[i].re); fields.push_back(fft->jcurrent[i].im);
        }
      }
      fft->update_conduct_order_param();
      rec.push_back(fft->condxinorm);
      rec.push_back(fft->condxiave);
      fft->prepare_next_conditr();
    }
    std::vector<double> out(fft->condxi[0], fft->condxi[0] + 2 * N);
    out.insert(out.end(), rec.begin(), rec.end());
    out.insert(out.end(), fields.begin(), fields.end());
    write_bin(cond_out, out.data(), out.size());
    fflush(stdout);
    MPI_Finalize();
    return 0;
  }
  double flops0 = pfdd_shim_fft_flops();
  auto t0 = std::chrono::steady_clock::now();
  app->iterate();
  auto t1 = std::chrono::steady_clock::now();
  double loop_s = std::chrono::duration<double>(t1 - t0).count();

  if (setup_out) {
    FILE *f = fopen(setup_out, "w");
    fprintf(f, "nx %d\nny %d\nnz %d\nS %d\n", fft->nx, fft->ny, fft->nz, S);
    fprintf(f, "CD %.17g\ntimestep %.17g\n", app->CD, app->timestep);
    fprintf(f, "C44 %.17g\nC12 %.17g\nC11 %.17g\n", mat->C44, mat->C12, mat->C11);
    fprintf(f, "mu %.17g\nxnu %.17g\nb %.17g\ndslip %.17g\n", mat->mu, mat->xnu, mat->b, mat->dslip);
    fprintf(f, "isf %.17g\nusf %.17g\nAn %.17g\n", mat->isf, mat->usf, mat->An);
    fprintf(f, "core_flag %d\n", app->core_flag);
    fprintf(f, "young %.17g\nC44in %.17g\n", mat->young, mat->C44);
    const double *cs[7] = {&mat->c0, &mat->c1, &mat->c2, &mat->c3, &mat->c4, &mat->a1, &mat->a3};
    for (int i = 0; i < 7; ++i) fprintf(f, "c%d %.17g\n", i, *cs[i]);
    const double *as[5] = {&mat->aa0, &mat->aa1, &mat->aa2, &mat->aa3, &mat->aa4};
    for (int i = 0; i < 5; ++i) fprintf(f, "aa%d %.17g\n", i, *as[i]);
    const double *bs[4] = {&mat->bb1, &mat->bb2, &mat->bb3, &mat->bb4};
    for (int i = 0; i < 4; ++i) fprintf(f, "bb%d %.17g\n", i + 1, *bs[i]);
    for (int a = 0; a < S; ++a)
      fprintf(f, "slip %d %.17g %.17g %.17g %.17g %.17g %.17g\n", a, fft->xn[a][0], fft->xn[a][1],
              fft->xn[a][2], fft->xb[a][0], fft->xb[a][1], fft->xb[a][2]);
    for (int a = 0; a < S; ++a) fprintf(f, "tau %d %.17g\n", a, fft->tau[a]);
    for (int i = 0; i < 3; ++i)
      fprintf(f, "four %d %.17g %.17g %.17g\n", i, fft->four[i][0], fft->four[i][1], fft->four[i][2]);
    for (int i = 0; i < 3; ++i)
      fprintf(f, "sigma_rot %d %.17g %.17g %.17g\n", i, fft->sigma_rot[i][0], fft->sigma_rot[i][1],
              fft->sigma_rot[i][2]);
    fprintf(f, "usfe_fit %.17g %.17g %.17g %.17g %.17g\n", mat->a_slope, mat->a_b, mat->b_b, mat->c_slope, mat->c_b);
    fprintf(f, "non_schmid %d %.17g %.17g %.17g %.17g\n", app->non_Schmid, app->angle_to_110, app->w1, app->w2,
            app->w3);
    fprintf(f, "iterations %zu\n", fft->step_xinorm.size());
    fclose(f);
  }
  if (state_out) write_bin(state_out, fft->xi[0], 2 * (size_t)S * N);
  if (B_out) write_bin(B_out, fft->BB, (size_t)S * S * N);
  if (stress_out) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        fft->local_sigma[i][j] = fft->avepst[i][j] = fft->avepsts[i][j] = fft->avepsd[i][j] = 0.0;
        fft->aveps[i][j] = fft->ave_eps[i][j] = fft->ave_sigma[i][j] = 0.0;
      }
    fft->prep_forward();
    fft->strain();
    fft->total_average_strain();
    fft->stress();
    std::vector<double> out;
    out.insert(out.end(), fft->data_eps, fft->data_eps + 2 * 9 * (size_t)N);
    out.insert(out.end(), fft->data_sigma, fft->data_sigma + 2 * 9 * (size_t)N);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out.push_back(fft->ave_eps[i][j]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out.push_back(fft->ave_sigma[i][j]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out.push_back(fft->avepst[i][j]);
    write_bin(stress_out, out.data(), out.size());
  }
  if (profile_out) {
    // FFTW_Slab::project_core_energy on the final state (data_fftw = xi after
    // prepare_next_itr): num_planes, delta [NP*N], then ddelta on the
    // j = ny/2, k = nz/2 line of each plane [NP*nx]
    fft->project_core_energy();
    const int NP = app->num_planes;
    const int n2 = fft->local_y, n3 = fft->local_z;
    std::vector<double> out;
    out.push_back((double)NP);
    out.insert(out.end(), fft->delta, fft->delta + (size_t)NP * N);
    for (int p = 0; p < NP; ++p)
      for (int i = 0; i < fft->nx; ++i)
        out.push_back(fft->ddelta[(size_t)p * N + (size_t)i * n2 * n3 + (size_t)(n2 / 2) * n3 + n3 / 2]);
    write_bin(profile_out, out.data(), out.size());
  }
  if (stats_out) {
    FILE *f = fopen(stats_out, "w");
    for (size_t i = 0; i < fft->step_xinorm.size(); ++i)
      fprintf(f, "%zu %.17g %.17g\n", i, fft->step_xinorm[i], fft->step_xiave[i]);
    fclose(f);
  }
  if (timing) {
    size_t iters = fft->step_xinorm.size();
    double upd = (double)S * (double)N * (double)iters;
    printf("{\"loop_s\": %.6f, \"iterations\": %zu, \"site_slip_updates_per_s\": %.6g, "
           "\"fft_gflops\": %.4f}\n",
           loop_s, iters, upd / loop_s, (pfdd_shim_fft_flops() - flops0) / loop_s * 1e-9);
  }
  fflush(stdout);
  // The reference never frees its fields (FFTW_Slab destructor is empty); skip
  // PFDD_C teardown the same way the process exit would.
  MPI_Finalize();
  return 0;
}
#endif  // PFDD_ORACLE_SLAB_ONLY
