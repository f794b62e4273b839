// Device kernels of the directional FMM matvec (sm_100a).
//
// Layout in HBM (all arrays indexed by expansion slot, see plan.hpp):
//   M[slot][LL], L[slot][LL]      multipole / local expansions (complex)
//   F[slot-f0][PP], J[slot-t0][PP] Fourier spectra of one cone batch
//   tables[t][PP]                 transfer spectra, perm[hash][PP] (uint16)
// Index order inside an expansion is the reference's (thetis_keys.hpp:35-53):
// i = (I0*L + I1)*L + I2, last axis fastest; spectra are P^3 row-major.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dfb {

// Most right-hand sides carried through one pass of the far and near field
// (expansions hold R = 1 .. kMaxRhsBlock vectors per slot).
constexpr int kMaxRhsBlock = 32;

template <typename T> struct cpx_t;
template <> struct cpx_t<double> { typedef double2 type; };
template <> struct cpx_t<float> { typedef float2 type; };

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C>
__device__ __forceinline__ C cmulc(C a, C b) {  // conj(a) * b
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.x * b.y - a.y * b.x;
  return r;
}
template <typename C>
__device__ __forceinline__ void cfma(C& acc, C a, C b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
template <typename C, typename R>
__device__ __forceinline__ void rfma(C& acc, R a, C b) {  // acc += a * b, a real
  acc.x = fma(a, b.x, acc.x);
  acc.y = fma(a, b.y, acc.y);
}
template <typename C>
__device__ __forceinline__ C czero() {
  C r;
  r.x = 0;
  r.y = 0;
  return r;
}

// Everything the kernels need about one operator, passed by value.
struct DevPlan {
  // trees
  const int32_t *S_first, *S_nprt, *S_lvl, *T_first, *T_nprt, *T_lvl, *T_parent;
  const double4 *S_ctr, *T_ctr;                // x, y, z, rad
  const double *S_pos, *T_pos;                 // 3 per particle, tree order
  const int32_t *S_perm, *T_perm;
  // slots
  const int32_t *sS_cell, *sS_dir, *sT_cell, *sT_dir;
  const int64_t *S_cptr, *T_cptr;              // per cell -> its slots (CSR)
  const int32_t *S_cslot, *S_cdir, *T_cslot, *T_cdir;
  // operators
  const int64_t *m2m_ptr, *l2l_ptr, *m2l_ptr;
  const int32_t *m2m_child, *l2l_parent, *m2l_src;
  const uint32_t* m2l_tab;
  const uint16_t* perm;
  const double* dirs;                          // all stages, 3 per direction
  int64_t dir_off[32];                         // per stage
  int64_t sig_off[32];                         // per stage, in complex elements
  int8_t ishf[32], hfstage[32];
  int* err;                                    // device flag: inconsistent list entry seen
  double kappa;
  int nlvl;
};

// Leaf slots of cell c (CSR of the slot lists, directions increasing) whose
// direction lies in [d0, d1): a contiguous sub-range [*b, *e).
__device__ __forceinline__ void dir_range(const int64_t* __restrict__ cptr, const int32_t* __restrict__ cdir,
                                          int64_t c, int d0, int d1, int64_t* b, int64_t* e) {
  int64_t lo = cptr[c], hi = cptr[c + 1];
  int64_t a = lo, z = hi;
  while (a < z) {  // first entry with dir >= d0
    const int64_t m = (a + z) >> 1;
    if (cdir[m] < d0) a = m + 1; else z = m;
  }
  int64_t a2 = a, z2 = hi;
  while (a2 < z2) {  // first entry with dir >= d1
    const int64_t m = (a2 + z2) >> 1;
    if (cdir[m] < d1) a2 = m + 1; else z2 = m;
  }
  *b = a;
  *e = a2;
}

}  // namespace dfb
