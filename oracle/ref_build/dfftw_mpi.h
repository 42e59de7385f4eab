/* FFTW 2.1.5 MPI-API stand-in used only to compile the reference PFDD sources
 * into a CPU oracle (test infrastructure).
 *
 * FFTW 2.1.5 is an external dependency of the reference (README.md "set-up to
 * use FFTW 2.1.5"; fft_fftw_slab.h:27) that is neither vendored nor installed
 * here.  This header keeps the names, argument order and semantics of the
 * calls the reference makes (fft_fftw_slab.cpp:66-68, 130-132, 1962, 1985,
 * 2021, 2043, 3386, 3424, 3466):
 *   - fftw_complex is {double re, im};
 *   - FFTW_FORWARD = -1 (exp(-2 pi i jk/n)), FFTW_BACKWARD = +1, both unnormalised;
 *   - fftwnd_mpi(plan, howmany, data, work, order) transforms in place,
 *     `howmany` fields interleaved with unit stride (element i of field f at
 *     data[i*howmany + f]);
 *   - with one rank the slab is the whole grid: local_nx = nx, start 0,
 *     total_local_size = nx*ny*nz.
 * The arithmetic behind it is a project-written FP64 mixed-radix Stockham FFT
 * (fftw2_shim.cpp), i.e. the published discrete Fourier transform, checked
 * against numpy.fft by tests/test_oracle_fft_shim.py.
 */
#ifndef PFDD_ORACLE_DFFTW_MPI_H
#define PFDD_ORACLE_DFFTW_MPI_H

#include "mpi.h"

typedef double fftw_real;
typedef struct { fftw_real re, im; } fftw_complex;

typedef enum { FFTW_FORWARD = -1, FFTW_BACKWARD = 1 } fftw_direction;
typedef enum { FFTW_NORMAL_ORDER, FFTW_TRANSPOSED_ORDER } fftwnd_mpi_output_order;

#define FFTW_ESTIMATE (0)
#define FFTW_MEASURE (1)

typedef struct pfdd_shim_plan3d *fftwnd_mpi_plan;

fftwnd_mpi_plan fftw3d_mpi_create_plan(MPI_Comm comm, int nx, int ny, int nz,
                                       fftw_direction dir, int flags);
void fftwnd_mpi_local_sizes(fftwnd_mpi_plan p, int *local_nx, int *local_x_start,
                            int *local_ny_after_transpose,
                            int *local_y_start_after_transpose,
                            int *total_local_size);
void fftwnd_mpi(fftwnd_mpi_plan p, int n_fields, fftw_complex *local_data,
                fftw_complex *work, fftwnd_mpi_output_order output_order);
void fftwnd_mpi_destroy_plan(fftwnd_mpi_plan p);

/* Shim-only extra (not part of FFTW 2): total flop-equivalent work done so far,
 * counted as 5 n log2 n per complex transform of length n, so a harness can
 * report the FFT rate of the baseline it times. */
extern "C" double pfdd_shim_fft_flops(void);

#endif
