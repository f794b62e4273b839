// Test infrastructure (oracle only): FFTW3-API shim used to compile the
// reference defmm here (FFTW3 is not installed).  The transform is the DFT by
// definition, applied axis by axis on row-major arrays, which is exact up to
// rounding for the odd sizes P = 2L-1 the reference uses (3..15).  Results
// match a genuine FFTW build only up to summation-order rounding, and the
// reference's M2F/F2L phase timings taken with this shim are those of a
// direct DFT, not of FFTW.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

struct oracle_fftw_plan_s {
  int rank;
  std::vector<int> n;
  int howmany;
  int idist, odist;
  int sign;
  fftw_complex* in;
  fftw_complex* out;
  // per distinct axis length: twiddles w[m] = exp(sign * 2 pi i m / len)
  std::vector<std::vector<std::complex<double>>> tw;
};

namespace {

typedef std::complex<double> cd;

std::vector<cd> twiddles(int len, int sign) {
  std::vector<cd> w(len);
  for (int m = 0; m < len; ++m) {
    long double a = 2.0L * 3.14159265358979323846264338327950288L *
                    (long double)m / (long double)len;
    w[m] = cd((double)cosl(a), (double)(sign * sinl(a)));
  }
  return w;
}

// In-place DFT of one multi-dimensional array (row-major).
void transform_one(const oracle_fftw_plan_s* p, cd* data) {
  long total = 1;
  for (int d = 0; d < p->rank; ++d) total *= p->n[d];
  std::vector<cd> line, res;
  long inner = 1;
  for (int d = p->rank - 1; d >= 0; --d) {
    const int len = p->n[d];
    const std::vector<cd>& w = p->tw[d];
    const long outer = total / ((long)len * inner);
    line.resize(len);
    res.resize(len);
    for (long o = 0; o < outer; ++o) {
      for (long i = 0; i < inner; ++i) {
        cd* base = data + o * (long)len * inner + i;
        for (int j = 0; j < len; ++j) line[j] = base[(long)j * inner];
        for (int k = 0; k < len; ++k) {
          cd acc(0.0, 0.0);
          int m = 0;
          for (int j = 0; j < len; ++j) {
            acc += line[j] * w[m];
            m += k;
            if (m >= len) m -= len;
          }
          res[k] = acc;
        }
        for (int k = 0; k < len; ++k) base[(long)k * inner] = res[k];
      }
    }
    inner *= len;
  }
}

oracle_fftw_plan_s* make_plan(int rank, const int* n, int howmany,
                              fftw_complex* in, int idist, fftw_complex* out,
                              int odist, int sign) {
  oracle_fftw_plan_s* p = new oracle_fftw_plan_s;
  p->rank = rank;
  p->n.assign(n, n + rank);
  p->howmany = howmany;
  p->idist = idist;
  p->odist = odist;
  p->sign = sign;
  p->in = in;
  p->out = out;
  for (int d = 0; d < rank; ++d) p->tw.push_back(twiddles(n[d], sign));
  return p;
}

void run(const oracle_fftw_plan_s* p, fftw_complex* in, fftw_complex* out) {
  long total = 1;
  for (int d = 0; d < p->rank; ++d) total *= p->n[d];
  std::vector<cd> buf(total);
  for (int b = 0; b < p->howmany; ++b) {
    const cd* src = reinterpret_cast<const cd*>(in) + (long)b * p->idist;
    cd* dst = reinterpret_cast<cd*>(out) + (long)b * p->odist;
    std::memcpy(buf.data(), src, sizeof(cd) * total);
    transform_one(p, buf.data());
    std::memcpy(dst, buf.data(), sizeof(cd) * total);
  }
}

}  // namespace

extern "C" {

fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in,
                        fftw_complex* out, int sign, unsigned) {
  long total = 1;
  for (int d = 0; d < rank; ++d) total *= n[d];
  return make_plan(rank, n, 1, in, (int)total, out, (int)total, sign);
}

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
                             fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed,
                             int ostride, int odist, int sign, unsigned) {
  // The reference only uses unit strides and no embedding beyond n.
  if (istride != 1 || ostride != 1) std::abort();
  (void)inembed;
  (void)onembed;
  return make_plan(rank, n, howmany, in, idist, out, odist, sign);
}

void fftw_execute(const fftw_plan p) { run(p, p->in, p->out); }

void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
  run(p, in, out);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
