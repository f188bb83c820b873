// Direct-summation DFTs behind the FFTW 3 stand-in interface of fftw3.h (see there).  Transforms of rank d
// over a row-major n[0] x ... x n[d-1] grid are done one axis at a time with a twiddle table per axis, in
// long double accumulation; r2c keeps the first n[d-1]/2+1 entries of the last axis, c2r rebuilds the full
// spectrum from Hermitian symmetry and returns the real part of the unnormalised inverse.  Test
// infrastructure only (the checker for the reference's FFT-based Lagrange M2L); sizes there are (2p-1)^3.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

typedef std::complex<long double> cld;

enum Kind { C2C, R2C, C2R };

struct Plan {
  Kind kind;
  bool single;  // float arrays
  int sign;
  std::vector<int> n;
  void *in, *out;
};

long long total(const std::vector<int> &n) {
  long long t = 1;
  for (int v : n) t *= v;
  return t;
}

// in-place transform of a full complex grid along every axis
void dft_grid(std::vector<cld> &a, const std::vector<int> &n, int sign) {
  const int d = (int)n.size();
  long long inner = 1;
  for (int ax = d - 1; ax >= 0; --ax) {
    const int m = n[ax];
    std::vector<cld> tw(m), line(m), res(m);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < m; ++k) {
      const long double ang = 2.0L * pi * (long double)k / (long double)m * (long double)sign;
      tw[k] = cld(std::cos(ang), std::sin(ang));
    }
    const long long outer = total(n) / ((long long)m * inner);
    for (long long o = 0; o < outer; ++o)
      for (long long i = 0; i < inner; ++i) {
        const long long base = o * m * inner + i;
        for (int j = 0; j < m; ++j) line[j] = a[base + j * inner];
        for (int k = 0; k < m; ++k) {
          cld s(0.0L, 0.0L);
          for (int j = 0; j < m; ++j) s += line[j] * tw[(long long)j * k % m];
          res[k] = s;
        }
        for (int k = 0; k < m; ++k) a[base + k * inner] = res[k];
      }
    inner *= m;
  }
}

template <class R>
void run(const Plan &p) {
  const long long N = total(p.n);
  const int last = p.n.back();
  const int half = last / 2 + 1;
  const long long rows = N / last;
  std::vector<cld> a(N);
  if (p.kind == C2C) {
    const R *in = (const R *)p.in;
    for (long long i = 0; i < N; ++i) a[i] = cld(in[2 * i], in[2 * i + 1]);
    dft_grid(a, p.n, p.sign);
    R *out = (R *)p.out;
    for (long long i = 0; i < N; ++i) {
      out[2 * i] = (R)a[i].real();
      out[2 * i + 1] = (R)a[i].imag();
    }
  } else if (p.kind == R2C) {
    const R *in = (const R *)p.in;
    for (long long i = 0; i < N; ++i) a[i] = cld(in[i], 0.0L);
    dft_grid(a, p.n, -1);
    R *out = (R *)p.out;
    for (long long r = 0; r < rows; ++r)
      for (int k = 0; k < half; ++k) {
        out[2 * (r * half + k)] = (R)a[r * last + k].real();
        out[2 * (r * half + k) + 1] = (R)a[r * last + k].imag();
      }
  } else {
    // full spectrum from the half one: X[idx] = conj(X[-idx mod n]) for the missing last-axis entries
    const R *in = (const R *)p.in;
    const int d = (int)p.n.size();
    std::vector<int> idx(d);
    for (long long f = 0; f < N; ++f) {
      long long rem = f;
      for (int ax = d - 1; ax >= 0; --ax) {
        idx[ax] = (int)(rem % p.n[ax]);
        rem /= p.n[ax];
      }
      bool conj = idx[d - 1] >= half;
      long long src = 0;
      for (int ax = 0; ax < d; ++ax) {
        const int v = conj ? (p.n[ax] - idx[ax]) % p.n[ax] : idx[ax];
        src = src * (ax == d - 1 ? half : p.n[ax]) + v;
      }
      const cld v(in[2 * src], in[2 * src + 1]);
      a[f] = conj ? std::conj(v) : v;
    }
    dft_grid(a, p.n, +1);
    R *out = (R *)p.out;
    for (long long i = 0; i < N; ++i) out[i] = (R)a[i].real();
  }
}

Plan *make(Kind k, bool single, int rank, const int *n, void *in, void *out, int sign) {
  Plan *p = new Plan;
  p->kind = k;
  p->single = single;
  p->sign = sign;
  p->n.assign(n, n + rank);
  p->in = in;
  p->out = out;
  return p;
}

template <class H>
H as_handle(Plan *p) {
  return reinterpret_cast<H>(p);
}
template <class H>
const Plan &as_plan(H p) {
  return *reinterpret_cast<const Plan *>(p);
}

}  // namespace

extern "C" {

void *fftw_malloc(size_t n) { return std::malloc(n ? n : 1); }
void fftw_free(void *p) { std::free(p); }
fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
  return as_handle<fftw_plan>(make(C2C, false, rank, n, in, out, sign));
}
fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned) {
  return as_handle<fftw_plan>(make(R2C, false, rank, n, in, out, -1));
}
fftw_plan fftw_plan_dft_c2r(int rank, const int *n, fftw_complex *in, double *out, unsigned) {
  return as_handle<fftw_plan>(make(C2R, false, rank, n, in, out, +1));
}
void fftw_execute(const fftw_plan p) { run<double>(as_plan(p)); }
void fftw_destroy_plan(fftw_plan p) { delete &as_plan(p); }

void *fftwf_malloc(size_t n) { return std::malloc(n ? n : 1); }
void fftwf_free(void *p) { std::free(p); }
fftwf_plan fftwf_plan_dft(int rank, const int *n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned) {
  return as_handle<fftwf_plan>(make(C2C, true, rank, n, in, out, sign));
}
fftwf_plan fftwf_plan_dft_r2c(int rank, const int *n, float *in, fftwf_complex *out, unsigned) {
  return as_handle<fftwf_plan>(make(R2C, true, rank, n, in, out, -1));
}
fftwf_plan fftwf_plan_dft_c2r(int rank, const int *n, fftwf_complex *in, float *out, unsigned) {
  return as_handle<fftwf_plan>(make(C2R, true, rank, n, in, out, +1));
}
void fftwf_execute(const fftwf_plan p) { run<float>(as_plan(p)); }
void fftwf_destroy_plan(fftwf_plan p) { delete &as_plan(p); }

}  // extern "C"
