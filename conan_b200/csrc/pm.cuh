// pm.cuh -- interfaces shared by the solver, initial-condition, adjoint and
// ensemble translation units.
#pragma once

#include "pm_kernels.cuh"
#include "profiler.cuh"

struct conan_pm;

namespace conan {

// Scale-factor rate adot(a) (Cosmology::operator(), src/run/cosmology.hh:16-23).
double adot(double H0, double Om, double OL, double a);
int check_pm_params(const conan_pm_params *p);
// Status of a kernel error word (CONAN_OK when 0): bit 3 (value 8), a
// bounded wait for a bulk copy that ran out, is CONAN_ERR_TIMEOUT; the
// other bits are failed self-checks of the deposit (CONAN_ERR_STATE).
int err_word_status(int h);
// Selects device `dev`, failing with a message when there is none.
int device_guard(int dev);

struct PMBase {
    virtual ~PMBase() {}
    virtual int init(const double *phi, double a_pos, double a_mom) = 0;
    virtual int drift(double a, double da) = 0;
    virtual int kick(double a, double da) = 0;
    virtual int run(conan_pm *h, const double *phi, double a0, double da, unsigned n, conan_step_cb cb,
                    void *user) = 0;
    virtual int get_state(double *X, double *P) = 0;
    virtual int set_state(const double *X, const double *P, double a_pos, double a_mom) = 0;
    virtual int density(double *out) = 0;
    virtual int potential(double *out) = 0;
    virtual int power_spectrum(int nbins, double *k, double *P, double *cnt) = 0;
    virtual int scale_factors(double *a_pos, double *a_mom) = 0;
    virtual int set_profiling(int on) = 0;
    virtual int profile_entry(int i, char *name, int *launches, double *ms) = 0;
    virtual int profile_reset() = 0;
    virtual int device_bytes(size_t *b) = 0;
    virtual int sync() = 0;
    virtual int set_cb_every(unsigned k) = 0;
    virtual int set_deposit(int mode) = 0;
    virtual int get_deposit(int *mode) = 0;
    virtual int autotune(double a, double da, char *report, size_t len) = 0;
    virtual int device() const = 0;
    virtual void *stream() const = 0;
};

PMBase *make_pm(const conan_pm_params &p);

// Shell-binned power spectrum of a half spectrum (see conan_pm_power_spectrum).
template <typename T>
int spectrum_bins(const typename Cplx<T>::type *spec, const Mesh &m, double L, int nbins, double *k,
                  double *Pk, double *cnt, cudaStream_t st, PMBase *unused);

}  // namespace conan
