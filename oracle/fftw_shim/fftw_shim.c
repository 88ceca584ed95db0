/* Project-written FP64 complex FFT behind the FFTW3 API subset in fftw3.h.
 *
 * Test infrastructure only (the oracle's FFT). Iterative radix-2
 * Cooley-Tukey per axis, twiddles evaluated directly as cos/sin(2*pi*k/n)
 * (no recurrence) so the rounding error stays O(eps * log2 n). Row-major
 * layout, last axis fastest, unnormalised, as FFTW documents for
 * fftw_plan_dft. Only power-of-two extents are accepted: the reference only
 * ever transforms boxes of 2^mbits per side (src/ic/main.cc:74,
 * src/run/main.cc:82-87).
 */
#include "fftw3.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

struct conan_shim_plan {
    int rank;
    int n[8];
    size_t total;
    double *in;
    double *out;
    int sign;
};

void *fftw_malloc(size_t n) { return malloc(n ? n : 1); }
void fftw_free(void *p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in,
                        fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    if (rank < 1 || rank > 8) {
        fprintf(stderr, "fftw shim: unsupported rank %d\n", rank);
        abort();
    }
    struct conan_shim_plan *p = calloc(1, sizeof *p);
    p->rank = rank;
    p->total = 1;
    for (int i = 0; i < rank; ++i) {
        if (!is_pow2(n[i])) {
            fprintf(stderr, "fftw shim: extent %d is not a power of two\n", n[i]);
            abort();
        }
        p->n[i] = n[i];
        p->total *= (size_t)n[i];
    }
    p->in = (double *)in;
    p->out = (double *)out;
    p->sign = sign;
    return p;
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

/* In-place radix-2 transform of one contiguous line of n complex values. */
static void fft_line(double *a, int n, int sign, const double *tw) {
    /* bit reversal */
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = a[2 * i], ti = a[2 * i + 1];
            a[2 * i] = a[2 * j];
            a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = tr;
            a[2 * j + 1] = ti;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1;
        int stride = n / len; /* twiddle index step into the size-n table */
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < half; ++k) {
                double wr = tw[2 * (k * stride)];
                double wi = sign * tw[2 * (k * stride) + 1];
                double *u = a + 2 * (s + k);
                double *v = a + 2 * (s + k + half);
                double xr = v[0] * wr - v[1] * wi;
                double xi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - xr;
                v[1] = u[1] - xi;
                u[0] += xr;
                u[1] += xi;
            }
        }
    }
}

void fftw_execute(const fftw_plan p) {
    if (p->out != p->in) memcpy(p->out, p->in, p->total * 2 * sizeof(double));
    double *data = p->out;
    size_t inner = p->total; /* product of extents after the current axis */
    for (int ax = 0; ax < p->rank; ++ax) {
        int n = p->n[ax];
        inner /= (size_t)n;
        size_t outer = p->total / ((size_t)n * inner);
        /* table of exp(-2 pi i k / n) for the forward sign */
        double *tw = malloc(sizeof(double) * 2 * (size_t)n);
        for (int k = 0; k < n; ++k) {
            double ang = -2.0 * M_PI * (double)k / (double)n;
            tw[2 * k] = cos(ang);
            tw[2 * k + 1] = sin(ang);
        }
        long long lines = (long long)(outer * inner);
#pragma omp parallel
        {
            double *line = malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(static)
            for (long long l = 0; l < lines; ++l) {
                size_t o = (size_t)l / inner, i = (size_t)l % inner;
                double *base = data + 2 * (o * (size_t)n * inner + i);
                for (int k = 0; k < n; ++k) {
                    line[2 * k] = base[2 * (size_t)k * inner];
                    line[2 * k + 1] = base[2 * (size_t)k * inner + 1];
                }
                fft_line(line, n, -p->sign, tw);
                for (int k = 0; k < n; ++k) {
                    base[2 * (size_t)k * inner] = line[2 * k];
                    base[2 * (size_t)k * inner + 1] = line[2 * k + 1];
                }
            }
            free(line);
        }
        free(tw);
    }
}
