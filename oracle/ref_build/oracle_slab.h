// Oracle-side subclass of the reference's FFTW_Slab numerics style.
// Test infrastructure only (links against the unmodified reference sources).
//
// It registers as `fft_style fftw_slab_oracle` and changes nothing in the
// arithmetic of the Ginzburg-Landau step.  It only
//   * sizes the gradient/core scratch arrays by max(slip_systems, num_planes):
//     FFTW_Slab::allocate (fft_fftw_slab.cpp:188-199) sizes them by num_planes,
//     but gradient() (fft_fftw_slab.cpp:869-1065) and core_energy_pyrII()
//     (fft_fftw_slab.cpp:1476-1484) write slip_systems*N entries;
//   * records xinorm / xiave after every update_order_parameter() call
//     (fft_fftw_slab.cpp:1746-1790) so the harness can write them out;
//   * with PFDD_ORACLE_SETUP_PROCS=P > 1 in the environment, runs the
//     reference's own per-wavevector set-up loops Bmatrix and Fmatrix
//     (fft_fftw_slab.cpp:466-638, 644-732) on P forked processes, each
//     calling them on one-x-plane slabs (local_x = 1, local_x_start = x, with
//     frec() for that slab) as an MPI run would on its slab, and writing into
//     shared mappings of BB / FF / DD.  The arithmetic per wavevector is the
//     reference's, so the tables are bit-identical to a one-process set-up;
//     only the set-up's wall time changes (a 256x256x128 grid with 12 systems
//     takes tens of minutes on one core).  The GL loop is not affected.
#ifdef FFT_CLASS
FftStyle(fftw_slab_oracle,OracleSlab)
#else

#ifndef PFDD_ORACLE_SLAB_H
#define PFDD_ORACLE_SLAB_H

#include <vector>
#include "fft_fftw_slab.h"

namespace PFDD_NS {

class OracleSlab : public FFTW_Slab {
 public:
  std::vector<double> step_xinorm, step_xiave;

  OracleSlab(class PFDD_C *p, int narg, char **arg) : FFTW_Slab(p, narg, arg) {}

  void allocate() override;
  void update_order_parameter() override;
  void Bmatrix() override;
  void Fmatrix() override;

 private:
  // (array member, components per wavevector) of one set-up table
  struct SlabOut {
    double **member;
    int comps;
  };
  // which = 0: FFTW_Slab::Bmatrix, 1: FFTW_Slab::Fmatrix (called non-virtually)
  void forked_setup(int which, SlabOut *outs, int nouts);
  void slab_call(int which);
};

}  // namespace PFDD_NS

#endif
#endif
