// Header-only C++ facade with the reference's public interface
// (IChollet/defmm include/interface.hpp:46-224) over the C ABI of
// libdefmm_b200.so (defmm_b200.h), so code written against the reference --
// e.g. its driver test/testinterface.cpp -- compiles unchanged:
//
//   IBFMM_Mat<3> A;  A.addSourceParticlesINP(..); A.addTargetParticlesINP(..);
//   A.prcmpt(L, Ncrit, kappa);  gemv(A, In, Out);  CheckFULL(A);
//
// Also provided, because the driver uses them: flt, cplx, cplx0, urand,
// Vecc (complex vector with operator[] and scalar assignment) and the colour
// constants f_cyan / f_def.  Errors throw std::runtime_error (the reference
// prints and calls exit(1)).  Link with -ldefmm_b200.
#ifndef DEFMM_B200_INTERFACE_HPP
#define DEFMM_B200_INTERFACE_HPP

#include <complex>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "defmm_b200.h"

typedef double flt;
typedef std::complex<flt> cplx;
const cplx cplx0 = cplx(0., 0.);
#ifndef urand
#define urand rand() / flt(RAND_MAX)
#endif
const char* const f_cyan = "\033[36m";
const char* const f_def = "\033[39m";
const char* const f_red = "\033[31m";

namespace defmm {

// Complex vector (the reference's gaia::Vec<cplx>, gaia_vectors.hpp).
class Vecc {
  std::vector<cplx> v_;

 public:
  Vecc() {}
  explicit Vecc(int n) : v_(n) {}
  const Vecc& operator=(const cplx& c) {
    for (auto& x : v_) x = c;
    return *this;
  }
  cplx& operator[](int i) { return v_[i]; }
  const cplx& operator[](int i) const { return v_[i]; }
  friend int Size(const Vecc& v) { return (int)v.v_.size(); }
  cplx* data() { return v_.data(); }
  const cplx* data() const { return v_.data(); }
};

template <int DIM>
class IBFMM_Mat {
  static_assert(DIM == 3, "defmm_b200 implements the 3-D operator");
  defmm_handle* h_;
  void check(int st) const {
    if (st) throw std::runtime_error(std::string("defmm_b200: ") + defmm_last_error(h_));
  }
  int64_t info(int what) const {
    int64_t v = 0;
    check(defmm_info(h_, what, &v));
    return v;
  }

 public:
  IBFMM_Mat() : h_(defmm_create()) {}
  ~IBFMM_Mat() { defmm_destroy(h_); }
  IBFMM_Mat(const IBFMM_Mat&) = delete;
  IBFMM_Mat& operator=(const IBFMM_Mat&) = delete;

  void addSourceParticle(flt part[DIM]) { check(defmm_add_source_particle(h_, part)); }
  void addTargetParticle(flt part[DIM]) { check(defmm_add_target_particle(h_, part)); }
  void addSourceParticlesINP(const char* name, int nparts) { check(defmm_load_inp(h_, name, nparts, 0)); }
  void addTargetParticlesINP(const char* name, int nparts) { check(defmm_load_inp(h_, name, nparts, 1)); }
  void prcmpt(int L, int Ncrit, flt kappa, int lvMAX = -1) { check(defmm_prcmpt(h_, L, Ncrit, kappa, lvMAX)); }
  // Not part of the reference: arithmetic of the matvec (DEFMM_PRECISION_*).
  void setPrecision(int mode) { check(defmm_set_precision(h_, mode)); }

  friend void gemv(IBFMM_Mat& A, Vecc& In, Vecc& Out) {
    A.check(defmm_gemv(A.h_, reinterpret_cast<const double*>(In.data()), reinterpret_cast<double*>(Out.data())));
  }

  // Sampled direct-sum check (2,000 seeded targets) printing the reference's
  // three relative norms (interface.hpp:218-220).
  friend void CheckFULL(IBFMM_Mat& A) {
    double err[3];
    A.check(defmm_check_full(A.h_, 2000, 7, err));
    std::cout << "Relative L^oo norm: " << f_cyan << err[0] << f_def << std::endl;
    std::cout << "Relative L^1  norm: " << f_cyan << err[1] << f_def << std::endl;
    std::cout << "Relative L^2  norm: " << f_cyan << err[2] << f_def << std::endl;
  }
};

}  // namespace defmm

#endif
