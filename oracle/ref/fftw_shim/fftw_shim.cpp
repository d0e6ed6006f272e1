// The FFTW_RODFT00 stand-in declared in fftw3.h (test infrastructure for
// oracle/_ref): the type-I discrete sine transform by direct sums, along the
// rows (n1, contiguous) and then the columns (n0) of the plan's array.
#include "fftw3.h"

#include <cmath>
#include <vector>

struct aprl_fftw_plan_s {
  int n0, n1;
  double* in;
  double* out;
  std::vector<double> sin0, sin1;  // sin(pi m / (n+1)) for m = 0 .. 2n+1
};

namespace {
// sin(pi m / (n + 1)) for every residue m of (j+1)(k+1) modulo 2(n+1).
std::vector<double> sine_table(int n) {
  const double pi = std::acos(-1.0);
  std::vector<double> t(2 * (n + 1));
  for (int m = 0; m < 2 * (n + 1); ++m) t[m] = std::sin(pi * m / (n + 1));
  return t;
}

// y[k] = 2 sum_j x[j * stride] sin(pi (j+1)(k+1) / (n+1)), k = 0 .. n-1.
void dst1(const double* x, double* y, int n, long stride, const std::vector<double>& table) {
  const long period = 2L * (n + 1);
  std::vector<double> result(n);
  for (int k = 0; k < n; ++k) {
    double sum = 0.0;
    for (int j = 0; j < n; ++j) sum += x[j * stride] * table[((long)(j + 1) * (k + 1)) % period];
    result[k] = 2.0 * sum;
  }
  for (int k = 0; k < n; ++k) y[k * stride] = result[k];
}
}  // namespace

extern "C" {

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double* in, double* out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, unsigned) {
  if (n0 < 1 || n1 < 1 || kind0 != FFTW_RODFT00 || kind1 != FFTW_RODFT00) return nullptr;
  aprl_fftw_plan_s* p = new aprl_fftw_plan_s;
  p->n0 = n0;
  p->n1 = n1;
  p->in = in;
  p->out = out;
  p->sin0 = sine_table(n0);
  p->sin1 = sine_table(n1);
  return p;
}

void fftw_execute(const fftw_plan p) {
  const long n1 = p->n1;
  if (p->out != p->in)
    for (long q = 0; q < (long)p->n0 * n1; ++q) p->out[q] = p->in[q];
  for (int r = 0; r < p->n0; ++r) dst1(p->out + r * n1, p->out + r * n1, p->n1, 1, p->sin1);
  for (int c = 0; c < p->n1; ++c) dst1(p->out + c, p->out + c, p->n0, n1, p->sin0);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
