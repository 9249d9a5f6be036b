// Separable O(n^4) DFT behind the FFTW plan API, for the pinning oracle build
// at test sizes (n <= 64). Test infrastructure only.
#include "fftw3-mpi.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <stdexcept>
#include <vector>

struct ns3d_fftw_plan_s {
    int n[3];
    fftw_complex *in;
    fftw_complex *out;
    int sign;
};

namespace {

// One 1-D DFT along `axis` of a row-major n0 x n1 x n2 complex array, in place.
void dft_axis(std::complex<double> *a, const int n[3], int axis, int sign) {
    const int len = n[axis];
    long stride = 1;
    for (int d = 2; d > axis; --d) stride *= n[d];
    std::vector<std::complex<double>> tw(len);
    for (int m = 0; m < len; ++m) {
        const double ang = sign * 2.0 * M_PI * (double)m / (double)len;
        tw[m] = std::complex<double>(std::cos(ang), std::sin(ang));
    }
    const long total = (long)n[0] * n[1] * n[2];
    std::vector<std::complex<double>> line(len), res(len);
    for (long base = 0; base < total; ++base) {
        // `base` must be the first element of a line along `axis`
        if ((base / stride) % len != 0) continue;
        for (int m = 0; m < len; ++m) line[m] = a[base + m * stride];
        for (int k = 0; k < len; ++k) {
            std::complex<double> s(0.0, 0.0);
            for (int m = 0; m < len; ++m) s += line[m] * tw[((long)k * m) % len];
            res[k] = s;
        }
        for (int k = 0; k < len; ++k) a[base + k * stride] = res[k];
    }
}

}  // namespace

extern "C" {

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned) {
    auto *p = new ns3d_fftw_plan_s;
    p->n[0] = n0; p->n[1] = n1; p->n[2] = n2;
    p->in = in; p->out = out; p->sign = sign;
    return p;
}

void fftw_execute(const fftw_plan p) {
    const long total = (long)p->n[0] * p->n[1] * p->n[2];
    auto *o = reinterpret_cast<std::complex<double> *>(p->out);
    auto *i = reinterpret_cast<std::complex<double> *>(p->in);
    if (o != i)
        for (long t = 0; t < total; ++t) o[t] = i[t];
    for (int axis = 0; axis < 3; ++axis) dft_axis(o, p->n, axis, p->sign);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
void *fftw_malloc(size_t n) { return std::malloc(n); }
void fftw_free(void *p) { std::free(p); }
fftw_complex *fftw_alloc_complex(size_t n) {
    return (fftw_complex *)std::malloc(n * sizeof(fftw_complex));
}

void fftw_mpi_init(void) { throw std::runtime_error("stub FFTW-MPI: not available"); }
void fftw_mpi_cleanup(void) {}
ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t, ptrdiff_t, ptrdiff_t, MPI_Comm, ptrdiff_t *,
                                 ptrdiff_t *) {
    throw std::runtime_error("stub FFTW-MPI: not available");
}
fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t, ptrdiff_t, ptrdiff_t, fftw_complex *, fftw_complex *,
                               MPI_Comm, int, unsigned) {
    throw std::runtime_error("stub FFTW-MPI: not available");
}

}  // extern "C"
