// fftw3.h -- TEST INFRASTRUCTURE ONLY: the one FFTW call of the reference's
// measurer (a 1-D real-to-complex forward transform, measurer.h:25-41), for the
// oracle's reference build.  A direct DFT in long double,
//   out[k] = sum_x in[x] exp(-2 pi i k x / n),  k = 0 .. n/2,
// FFTW's forward sign and its unnormalised convention.
#pragma once

#include <cmath>
#include <cstddef>

typedef double fftw_complex[2];
struct lgvshim_fftw_plan {
  int n;
  double *in;
  fftw_complex *out;
};
typedef lgvshim_fftw_plan *fftw_plan;
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

inline fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned) {
  return new lgvshim_fftw_plan{n, in, out};
}
inline void fftw_execute(const fftw_plan p) {
  const int n = p->n;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int k = 0; k <= n / 2; ++k) {
    long double re = 0.0L, im = 0.0L;
    for (int x = 0; x < n; ++x) {
      const long double ang = two_pi * (long double)(((long long)k * x) % n) / (long double)n;
      re += (long double)p->in[x] * cosl(ang);
      im -= (long double)p->in[x] * sinl(ang);
    }
    p->out[k][0] = (double)re;
    p->out[k][1] = (double)im;
  }
}
inline void fftw_destroy_plan(fftw_plan p) { delete p; }
