/* fft_b200.h -- the FFT style `b200`: the reference's FFT style object with
 * its Ginzburg-Landau iteration moved to libpfdd_b200.so.
 *
 * A maintainer drops this file and fft_b200.cpp (and solve_GLgpu.{h,cpp})
 * into the reference's src/, regenerates the style headers and links
 * -lpfdd_b200.  It registers like every FFT style (FftStyle, as
 * src/fft_fftw_slab.h:16-17; instantiated by Input::fft_style,
 * src/input.cpp:693-708) and keeps FFTW_Slab for everything off the GL hot
 * path: decks, initial conditions (initial_sxtal_*), resolved shear stress for
 * the host's prints, dumps and diagnostics.  Deck syntax: the fftw_slab
 * arguments plus
 *     precision fp64|fp32   arithmetic of the GPU step (default fp64)
 *     diag host|gpu         strain/stress at output steps: `host` runs the
 *                           reference's own strain()/stress() on the state
 *                           pair the reference's loop holds there (exact);
 *                           `gpu` uses pfdd_gpu_strain_stress on the current
 *                           state and skips the host B(k)/F(k) tables
 * e.g.  fft_style b200 pbc 1 1 1 mode 1 precision fp32 diag gpu
 */
#ifdef FFT_CLASS
FftStyle(b200,FFT_B200)
#else

#ifndef PFDD_FFT_B200_H
#define PFDD_FFT_B200_H

#include <vector>

#include "fft_fftw_slab.h"
#include "pfdd_b200.h"

namespace PFDD_NS {

class FFT_B200 : public FFTW_Slab {
 public:
  // the fftw_slab arguments without this style's own keywords (the FFT base
  // constructor rejects words it does not know, src/fft.cpp:92-151)
  struct StyleArgs {
    std::vector<char *> rest;
    int precision, diag_gpu, bad;
    StyleArgs(int narg, char **arg);
  };
  FFT_B200(class PFDD_C *, int, char **);
  FFT_B200(class PFDD_C *, StyleArgs &&);
  ~FFT_B200();

  // FFTW_Slab::allocate, after giving App::num_planes a defined value where
  // the app left it unset (e.g. app_2d_bcc_ortho_1loop.cpp never sets it;
  // allocate sizes the gradient arrays by it, fft_fftw_slab.cpp:140-199)
  void allocate() override;

  // FFTW_Slab::setup (src/fft_fftw_slab.cpp:111-119), then the device handle
  // from the members the reference holds after App::init / set_slip
  void setup() override;

  // with `diag gpu`: the strain/stress diagnostics (src/fft_fftw_slab.cpp:
  // 3252-3553, called by DiagStress::compute and DumpText) from the GPU
  void strain() override;
  void total_average_strain() override;
  void stress() override;

  pfdd_gpu *gpu;
  int precision;    // PFDD_FP64 / PFDD_FP32
  int diag_gpu;     // 1: strain/stress from pfdd_gpu_strain_stress
  int diag_fresh;   // the GPU diagnostics of the current output step are in place

  // The GL iterations of SolveGLGPU: `n` steps at the current stress state
  // with the tolerance test; returns the device's record.
  pfdd_step_stats advance(int n, double tol);
  void set_device_stress();   // this stress state's sigma (App::sigma) on the device
  void pull_xi();             // xi[0] <- device state (reference interleaved layout)
  void push_xi();             // device state <- xi[0]

 private:
  void check(int status, const char *what);
  void gpu_diagnostics();
};

}  // namespace PFDD_NS

#endif
#endif
