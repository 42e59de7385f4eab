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
//     (fft_fftw_slab.cpp:1746-1790) so the harness can write them out.
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
};

}  // namespace PFDD_NS

#endif
#endif
