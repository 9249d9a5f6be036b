/*
 * FFTW-MPI declarations for the pinning oracle build. The reference calls these
 * only from compute_correlations_fftw (ana_isotropic.cpp:34-191), whose single
 * call site is commented out; the stand-ins throw if ever reached.
 */
#ifndef NS3D_ORACLE_FFTW3_MPI_STUB_H
#define NS3D_ORACLE_FFTW3_MPI_STUB_H

#include <stddef.h>
#include "fftw3.h"
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

void fftw_mpi_init(void);
void fftw_mpi_cleanup(void);
ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start);
fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in,
                               fftw_complex *out, MPI_Comm comm, int sign, unsigned flags);

#ifdef __cplusplus
}
#endif

#endif
