/*
 * Minimal FFTW3 API stand-in used ONLY to compile the reference's sources into
 * the pinning oracle (oracle/_ref). Test infrastructure, not product.
 * fftw_plan_dft_3d is served by a plain separable DFT (fftw_stub.cpp) with
 * FFTW's conventions: row-major n0 x n1 x n2, unnormalised,
 * FFTW_FORWARD = -1 (e^{-i...}), FFTW_BACKWARD = +1.
 */
#ifndef NS3D_ORACLE_FFTW3_STUB_H
#define NS3D_ORACLE_FFTW3_STUB_H

#include <stddef.h>

typedef double fftw_complex[2];
typedef struct ns3d_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD  (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

#ifdef __cplusplus
extern "C" {
#endif

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_complex *fftw_alloc_complex(size_t n);

#ifdef __cplusplus
}
#endif

#endif
