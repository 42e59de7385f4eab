/* solve_GLgpu.cpp -- solve style `GLgpu` (see solve_GLgpu.h). */
#include "solve_GLgpu.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "app.h"
#include "error.h"
#include "fft.h"
#include "fft_b200.h"
#include "output.h"
#include "timer.h"

using namespace PFDD_NS;

SolveGLGPU::SolveGLGPU(PFDD_C *pfdd_p, int narg, char **arg) : Solve(pfdd_p, narg, arg) {
  if (narg < 1) error->all(FLERR, "Illegal solve command");
  it = 0;
  max_iter = 10;
  sstate = 0;
  tol = 0.0;
  int iarg = 1;
  while (iarg < narg) {   // the keywords of SolveGL (src/solve_GL.cpp:44-56)
    if (!strcmp(arg[iarg], "max_iter") && iarg + 1 < narg) {
      max_iter = atoi(arg[iarg + 1]);
      iarg += 2;
    } else if (!strcmp(arg[iarg], "tol") && iarg + 1 < narg) {
      tol = atof(arg[iarg + 1]);
      iarg += 2;
    } else {
      error->all(FLERR, "Illegal solve_style GLgpu command");
    }
  }
}

SolveGLGPU::~SolveGLGPU() {}

// SolveGL::iterate (src/solve_GL.cpp:70-158).  Per stress state: tau for the
// host's prints, sigma on the device, then chunks of GL iterations ending at
// the next output step.  At an output step the host holds what the
// reference's loop holds there: xi after the step and, for the host
// diagnostics, data_fftw = FFT of the state before it (prep_forward) and the
// core profile of that state (project_core_energy, run after the previous
// step's prepare_next_itr).
void SolveGLGPU::iterate() {
  FFT_B200 *g = dynamic_cast<FFT_B200 *>(fft);
  if (!g) error->all(FLERR, "solve_style GLgpu needs fft_style b200");
  const int ND = app->dimension;
  const int stopsteps = app->stopsteps;
  timer->stamp();
  if (me == 0) printf("Beginning Time Evolution\n");
  bool leave = false;
  for (sstate = 0; sstate < stopsteps && !leave; sstate++) {
    fft->rotate_stress();
    app->resolSS();
    int done_it = 0;
    while (done_it < max_iter) {
      // iterations until the next output: the first with time >= nextoutput, or the last
      int k = 1;
      if (app->time < app->nextoutput) k = (int)std::ceil(app->nextoutput - app->time) + 1;
      if (k > max_iter - done_it) k = max_iter - done_it;
      if (k > 1) {
        const pfdd_step_stats st = g->advance(k - 1, tol);
        done_it += st.steps_done;
        app->time += st.steps_done;
        if (st.converged) {
          // the tolerance stopped the chunk: report at the converged state (its
          // last change is below tol; the host diagnostics transform that state)
          g->pull_xi();
          fft->prepare_next_itr();
          if (app->non_Schmid) fft->project_core_energy();
          if (!g->diag_gpu) fft->prep_forward();
          if (me == 0) printf("printing output it %d\n", done_it - 1);
          app->nextoutput = output->compute(app->time - 1, 1);
          if (me == 0) printf("Loading step %d converged after %d iterations\n", sstate, done_it - 1);
          break;
        }
      }
      // the output step
      if (!g->diag_gpu) {
        g->pull_xi();
        fft->prepare_next_itr();
        if (app->non_Schmid) fft->project_core_energy();
        fft->prep_forward();
      }
      const pfdd_step_stats st = g->advance(1, tol);
      g->pull_xi();
      if (g->diag_gpu && app->non_Schmid) {   // the core profile of the current state
        fft->prepare_next_itr();
        fft->project_core_energy();
      }
      const int itn = done_it;
      done_it += 1;
      const int last = st.converged || done_it == max_iter;
      if (last) {
        if (me == 0) printf("printing output it %d\n", itn);
        app->nextoutput = output->compute(app->time, 1);
      } else if (app->time >= app->nextoutput) {
        app->nextoutput = output->compute(app->time, 0);
      }
      timer->stamp(TIME_OUTPUT);
      timer->stamp(TIME_FFT);
      app->time++;
      if (st.converged) {
        if (me == 0) printf("Loading step %d converged after %d iterations\n", sstate, itn);
        break;
      }
    }
    for (int i = 0; i < ND; i++)
      for (int j = 0; j < ND; j++) fft->sigma[i][j] = fft->sigma[i][j] + fft->deltasig[i][j];
  }
  timer->stamp(TIME_SOLVE);
}
