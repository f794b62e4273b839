// Driver written against the reference's interface (the same calls as the
// reference's test/testinterface.cpp): INP input, prcmpt, gemv, CheckFULL.
// Built against include/interface.hpp (the defmm_b200 facade).
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "interface.hpp"

using namespace defmm;

int main(int argc, char* argv[]) {
  const char* inp = argc > 1 ? argv[1] : "points.inp";
  const int ORDER = argc > 2 ? atoi(argv[2]) : 4;
  const int NCRIT = argc > 3 ? atoi(argv[3]) : 32;
  const int N = 8000;
  // points on the unit sphere (deterministic), written as an INP file
  FILE* f = std::fopen(inp, "w");
  srand(1);
  for (int i = 0; i < N; i++) {
    double z = 2. * urand - 1., t = 2. * M_PI * urand, r = std::sqrt(1. - z * z);
    std::fprintf(f, "%.17g %.17g %.17g\n", r * std::cos(t), r * std::sin(t), z);
  }
  std::fclose(f);
  IBFMM_Mat<3> A;
  A.addSourceParticlesINP(inp, N);
  A.addTargetParticlesINP(inp, N);
  Vecc In(N), Out(N);
  Out = cplx0;
  for (int n = 0; n < N; n++) In[n] = cplx(urand);
  A.prcmpt(ORDER, NCRIT, 2. * M_PI * 6.);
  gemv(A, In, Out);
  CheckFULL(A);
  return 0;
}
