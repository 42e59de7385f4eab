/* solve_GLgpu.h -- the solve style `GLgpu`: SolveGL::iterate
 * (src/solve_GL.cpp:70-158) with its GL iterations run by libpfdd_b200.so
 * through the FFT style `b200` (fft_b200.h).
 *
 * Same deck arguments as `GL` (max_iter, tol) and the same control flow:
 * stress states, output when App::time reaches App::nextoutput or the state
 * ends (tolerance, last iteration), sigma += deltasig after each state.  The
 * iterations between two outputs run as one pfdd_gpu_advance call (CUDA-graph
 * replays on the device); the host only sees the state at output steps.
 *     solve_style GLgpu max_iter 5000 tol 1e-4
 */
#ifdef SOLVE_CLASS
SolveStyle(GLgpu,SolveGLGPU)
#else

#ifndef PFDD_SOLVE_GLGPU_H
#define PFDD_SOLVE_GLGPU_H

#include "solve.h"

namespace PFDD_NS {

class SolveGLGPU : public Solve {
 public:
  SolveGLGPU(class PFDD_C *, int, char **);
  ~SolveGLGPU();
  void iterate();
};

}  // namespace PFDD_NS

#endif
#endif
