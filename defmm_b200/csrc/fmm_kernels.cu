// Matvec kernels.  One template per phase, instantiated per precision (T)
// and interpolation order (L).  See kernels.cuh for the memory layout.
#include "kernels.cuh"
#include "fmm_kernels.h"

namespace dfb {

// ----------------------------------------------------------------- basics --
// equispaced Lagrange basis of order L on [-rad, rad] at x
// (thetis_polynomials.hpp:81-94): b[l] = prod_{j != l} (x/rad - p_j)/(p_l - p_j),
// p_j = -1 + 2 j/(L-1)
template <int L, typename T>
__device__ __forceinline__ void lagrange_all(T x, T rad, T* b) {
  const T nx = x / rad;
#pragma unroll
  for (int l = 0; l < L; l++) {
    T r = 1;
    const T pl = T(-1) + T(2) * (T(l) / T(L - 1));
#pragma unroll
    for (int j = 0; j < L; j++) {
      if (j == l) continue;
      const T pj = T(-1) + T(2) * (T(j) / T(L - 1));
      r *= (nx - pj) / (pl - pj);
    }
    b[l] = r;
  }
}

// exp(i a) with a in FP64 (argument reduction and evaluation by CUDA's sincos)
template <typename C>
__device__ __forceinline__ C expi64(double a) {
  double s, c;
  sincos(a, &s, &c);
  C r;
  r.x = c;
  r.y = s;
  return r;
}

// ------------------------------------------------------------- gather/scatter
template <typename T>
__global__ void k_gather(const double2* __restrict__ qin, const int32_t* __restrict__ perm,
                         typename cpx_t<T>::type* __restrict__ q, int64_t n, int64_t nrhs_stride_in,
                         int64_t nrhs_stride_q, int nrhs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t u = perm[i];
  for (int r = 0; r < nrhs; r++) {
    const double2 v = qin[r * nrhs_stride_in + u];
    typename cpx_t<T>::type w;
    w.x = (T)v.x;
    w.y = (T)v.y;
    q[r * nrhs_stride_q + i] = w;
  }
}

__global__ void k_scatter(const double2* __restrict__ pnear, const double2* __restrict__ pfar,
                          const int32_t* __restrict__ perm, double2* __restrict__ out, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 a = pnear[i], b = pfar[i];
  a.x += b.x;
  a.y += b.y;
  out[perm[i]] = a;
}

// -------------------------------------------------------------------- P2M --
// One CTA (4 warps) per source leaf at a precomputed level (upwpass.hpp:39-47).
// HF leaf (phfP2M, P2M.hpp:114-131), per effective direction d:
//   M_d[l] = conj(sig2_d[l]) * sum_j Z(l, j) exp(-i k d.(y_j - c)) q_j
// LF leaf (plfP2M, P2M.hpp:134-136): M[l] = sum_j Z(l, j) q_j,
// with Z(l, j) = prod_k S_{I_k(l)}(y_jk - c_k) the leaf's interpolation matrix
// (mapOnTrees.hpp:37-83).
template <typename T, int L>
__global__ void __launch_bounds__(128) k_p2m(DevPlan P, const int32_t* __restrict__ leaves, int nleaves,
                                             const typename cpx_t<T>::type* __restrict__ q,
                                             const typename cpx_t<T>::type* __restrict__ sig2,
                                             typename cpx_t<T>::type* __restrict__ M) {
  typedef typename cpx_t<T>::type C;
  constexpr int LL = L * L * L;
  constexpr int NPB = 64;
  __shared__ T Bs[NPB][3][L];
  __shared__ C wq[4][NPB];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int li = blockIdx.x; li < nleaves; li += gridDim.x) {
    const int c = leaves[li];
    const int n = P.S_nprt[c], f = P.S_first[c];
    const double4 ct = P.S_ctr[c];
    const int lv = P.S_lvl[c];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const int64_t sb = P.S_cptr[c], se = P.S_cptr[c + 1];
    const double* dirs = P.dirs + P.dir_off[h] * 3;
    const C* s2 = sig2 + P.sig_off[h];
    for (int p0 = 0; p0 < n; p0 += NPB) {
      const int np = min(NPB, n - p0);
      __syncthreads();
      for (int o = threadIdx.x; o < 3 * np; o += blockDim.x) {
        const int p = o / 3, k = o % 3;
        const double x = P.S_pos[3 * (int64_t)(f + p0 + p) + k] - (&ct.x)[k];
        T b[L];
        lagrange_all<L, T>((T)x, (T)ct.w, b);
#pragma unroll
        for (int l = 0; l < L; l++) Bs[p][k][l] = b[l];
      }
      __syncthreads();
      for (int64_t j = sb + warp; j < se; j += 4) {
        const int slot = P.S_cslot[j], d = P.S_cdir[j];
        for (int p = lane; p < np; p += 32) {
          C w = q[f + p0 + p];
          if (hf) {
            const double* y = P.S_pos + 3 * (int64_t)(f + p0 + p);
            const double* dv = dirs + 3 * d;
            double dp = 0.;
            for (int k = 0; k < 3; k++) dp += dv[k] * (y[k] - (&ct.x)[k]);
            C e = expi64<C>(-P.kappa * dp);
            w = cmul(w, e);
          }
          wq[warp][p] = w;
        }
        __syncwarp();
        for (int l = lane; l < LL; l += 32) {
          const int i0 = l / (L * L), i1 = (l / L) % L, i2 = l % L;
          C acc = czero<C>();
          for (int p = 0; p < np; p++) {
            const T z = Bs[p][0][i0] * Bs[p][1][i1] * Bs[p][2][i2];
            rfma(acc, z, wq[warp][p]);
          }
          if (hf) acc = cmulc(s2[(int64_t)d * LL + l], acc);
          C* out = M + (int64_t)slot * LL + l;
          if (p0 == 0) {
            *out = acc;
          } else {
            C o = *out;
            o.x += acc.x;
            o.y += acc.y;
            *out = o;
          }
        }
        __syncwarp();
      }
    }
  }
}

// ------------------------------------------------ separable 3-D transfer --
// out[a,b,c] = sum A_s0(a,a') A_s1(b,b') A_s2(c,c') in[a',b',c'] computed in
// three axis passes (axis 2, 1, 0 as interpolation.hpp:311-361); A(k, p) is
// stored column-major mat[k + p*L].  One warp, values l = lane + 32 m.
template <typename T, int L>
__device__ __forceinline__ void separable_warp(const T* mats, int sg0, int sg1, int sg2,
                                               typename cpx_t<T>::type* buf,
                                               typename cpx_t<T>::type* buf2,
                                               typename cpx_t<T>::type* res, int lane) {
  typedef typename cpx_t<T>::type C;
  constexpr int LL = L * L * L, NL = (LL + 31) / 32;
  const T* m2 = mats + sg2 * L * L;
  const T* m1 = mats + sg1 * L * L;
  const T* m0 = mats + sg0 * L * L;
#pragma unroll
  for (int m = 0; m < NL; m++) {
    const int l = lane + 32 * m;
    if (l < LL) {
      const int a = l / (L * L), b = (l / L) % L, c = l % L;
      C acc = czero<C>();
#pragma unroll
      for (int p = 0; p < L; p++) rfma(acc, m2[c + p * L], buf[(a * L + b) * L + p]);
      buf2[l] = acc;
    }
  }
  __syncwarp();
#pragma unroll
  for (int m = 0; m < NL; m++) {
    const int l = lane + 32 * m;
    if (l < LL) {
      const int a = l / (L * L), b = (l / L) % L, c = l % L;
      C acc = czero<C>();
#pragma unroll
      for (int p = 0; p < L; p++) rfma(acc, m1[b + p * L], buf2[(a * L + p) * L + c]);
      buf[l] = acc;
    }
  }
  __syncwarp();
#pragma unroll
  for (int m = 0; m < NL; m++) {
    const int l = lane + 32 * m;
    if (l < LL) {
      const int a = l / (L * L), b = (l / L) % L, c = l % L;
      C acc = czero<C>();
#pragma unroll
      for (int p = 0; p < L; p++) rfma(acc, m0[a + p * L], buf[(p * L + b) * L + c]);
      res[m] = acc;
    }
  }
  __syncwarp();
}

// -------------------------------------------------------------------- M2M --
// One warp per parent slot with children (upwpass.hpp:49-60):
//   HF parent, direction d (hfM2Mblock M2M.hpp:76-105 / lf2hfM2M :108-124):
//     M_d = conj(sig2_d) o sum_c exp(-i k d.v_c) A_{v_c}(sig_d o M_c)
//   LF parent (lfM2M :35-41): M = sum_c A_{v_c}(M_c);   v_c = ctr_c - ctr_parent
template <typename T, int L>
struct XferCfg {
  // warps per CTA so that 2 LL-vectors per warp fit in 40 KB of shared memory
  static constexpr int NW = (2 * L * L * L * (int)sizeof(typename cpx_t<T>::type) * 4 <= 40960) ? 4 : 2;
};

template <typename T, int L>
__global__ void __launch_bounds__(128) k_m2m(DevPlan P, int64_t s0, int64_t s1,
                                             const typename cpx_t<T>::type* __restrict__ sig,
                                             const typename cpx_t<T>::type* __restrict__ sig2,
                                             typename cpx_t<T>::type* __restrict__ M) {
  typedef typename cpx_t<T>::type C;
  constexpr int LL = L * L * L, NL = (LL + 31) / 32, NW = XferCfg<T, L>::NW;
  __shared__ T mats[2 * L * L];
  __shared__ C sbuf[NW][2][LL];
  for (int i = threadIdx.x; i < 2 * L * L; i += blockDim.x) mats[i] = (T)P.mats[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t ps = s0 + blockIdx.x * NW + warp; ps < s1; ps += (int64_t)gridDim.x * NW) {
    const int64_t eb = P.m2m_ptr[ps], ee = P.m2m_ptr[ps + 1];
    if (eb == ee) continue;  // leaf slot: written by P2M
    const int pc = P.sS_cell[ps], d = P.sS_dir[ps];
    const int lv = P.S_lvl[pc];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const double4 pct = P.S_ctr[pc];
    const C* sg = sig + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
    const C* sg2 = sig2 + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
    double dv[3] = {0., 0., 0.};
    if (hf)
      for (int k = 0; k < 3; k++) dv[k] = P.dirs[3 * (P.dir_off[h] + d) + k];
    C acc[NL];
#pragma unroll
    for (int m = 0; m < NL; m++) acc[m] = czero<C>();
    for (int64_t e = eb; e < ee; e++) {
      const int cs = P.m2m_child[e];
      const int cc = P.sS_cell[cs];
      const double4 cct = P.S_ctr[cc];
      const double v[3] = {cct.x - pct.x, cct.y - pct.y, cct.z - pct.z};
      const C* Mc = M + (int64_t)cs * LL;
      for (int l = lane; l < LL; l += 32) sbuf[warp][0][l] = hf ? cmul(sg[l], Mc[l]) : Mc[l];
      __syncwarp();
      C res[NL];
      separable_warp<T, L>(mats, v[0] < 0. ? 0 : 1, v[1] < 0. ? 0 : 1, v[2] < 0. ? 0 : 1,
                           sbuf[warp][0], sbuf[warp][1], res, lane);
      if (hf) {
        const C ph = expi64<C>(-P.kappa * (dv[0] * v[0] + dv[1] * v[1] + dv[2] * v[2]));
#pragma unroll
        for (int m = 0; m < NL; m++) cfma(acc[m], ph, res[m]);
      } else {
#pragma unroll
        for (int m = 0; m < NL; m++) {
          acc[m].x += res[m].x;
          acc[m].y += res[m].y;
        }
      }
    }
#pragma unroll
    for (int m = 0; m < NL; m++) {
      const int l = lane + 32 * m;
      if (l < LL) M[ps * LL + l] = hf ? cmulc(sg2[l], acc[m]) : acc[m];
    }
  }
}

// -------------------------------------------------------------------- L2L --
// One warp per child slot with parents (dwnpass.hpp:49-58):
//   HF parent direction d (hfL2Lblock L2L.hpp:78-108 / hf2lfL2L :111-127):
//     L_c += sum_d exp(i k v.d) conj(sig_d) o B_v(sig2_d o L_d)
//   LF parent (lfL2L :35-41): L_c += B_v(L_p);   v = ctr_child - ctr_parent
template <typename T, int L>
__global__ void __launch_bounds__(128) k_l2l(DevPlan P, int64_t s0, int64_t s1,
                                             const typename cpx_t<T>::type* __restrict__ sig,
                                             const typename cpx_t<T>::type* __restrict__ sig2,
                                             typename cpx_t<T>::type* __restrict__ Lx) {
  typedef typename cpx_t<T>::type C;
  constexpr int LL = L * L * L, NL = (LL + 31) / 32, NW = XferCfg<T, L>::NW;
  __shared__ T mats[2 * L * L];
  __shared__ C sbuf[NW][2][LL];
  for (int i = threadIdx.x; i < 2 * L * L; i += blockDim.x) mats[i] = (T)P.mats[2 * L * L + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t cs = s0 + blockIdx.x * NW + warp; cs < s1; cs += (int64_t)gridDim.x * NW) {
    const int64_t eb = P.l2l_ptr[cs], ee = P.l2l_ptr[cs + 1];
    if (eb == ee) continue;
    const int cc = P.sT_cell[cs];
    const int pc = P.T_parent[cc];
    const int lv = P.T_lvl[pc];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const double4 pct = P.T_ctr[pc], cct = P.T_ctr[cc];
    const double v[3] = {cct.x - pct.x, cct.y - pct.y, cct.z - pct.z};
    const int sg0 = v[0] < 0. ? 0 : 1, sg1 = v[1] < 0. ? 0 : 1, sg2i = v[2] < 0. ? 0 : 1;
    C acc[NL];
#pragma unroll
    for (int m = 0; m < NL; m++) acc[m] = czero<C>();
    for (int64_t e = eb; e < ee; e++) {
      const int ps = P.l2l_parent[e];
      const int d = P.sT_dir[ps];
      const C* Lp = Lx + (int64_t)ps * LL;
      const C* sg = sig + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
      const C* sgq = sig2 + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
      for (int l = lane; l < LL; l += 32) sbuf[warp][0][l] = hf ? cmul(sgq[l], Lp[l]) : Lp[l];
      __syncwarp();
      C res[NL];
      separable_warp<T, L>(mats, sg0, sg1, sg2i, sbuf[warp][0], sbuf[warp][1], res, lane);
      if (hf) {
        const double* dv = P.dirs + 3 * (P.dir_off[h] + d);
        const C ph = expi64<C>(P.kappa * (v[0] * dv[0] + v[1] * dv[1] + v[2] * dv[2]));
#pragma unroll
        for (int m = 0; m < NL; m++) {
          const int l = lane + 32 * m;
          if (l < LL) cfma(acc[m], ph, cmulc(sg[l], res[m]));
        }
      } else {
#pragma unroll
        for (int m = 0; m < NL; m++) {
          acc[m].x += res[m].x;
          acc[m].y += res[m].y;
        }
      }
    }
#pragma unroll
    for (int m = 0; m < NL; m++) {
      const int l = lane + 32 * m;
      if (l < LL) {
        C o = Lx[cs * LL + l];
        o.x += acc[m].x;
        o.y += acc[m].y;
        Lx[cs * LL + l] = o;
      }
    }
  }
}

// ---------------------------------------------------------------- M2F/F2L --
// Pruned odd-size 3-D DFT (size P = 2L-1) of the zero-padded expansion
// (circulant.hpp:96-106: M sits at the low corner of the P^3 grid):
//   F[k0,k1,k2] = sum_{a,b,c<L} M[a,b,c] w^(k0 a + k1 b + k2 c),  w = e^{-2 pi i/P}
template <typename T, int L>
__global__ void k_m2f(int64_t n, const typename cpx_t<T>::type* __restrict__ M,
                      typename cpx_t<T>::type* __restrict__ F) {
  typedef typename cpx_t<T>::type C;
  constexpr int P = 2 * L - 1, LL = L * L * L, PP = P * P * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* W = reinterpret_cast<C*>(smem_raw);
  C* Mi = W + P;
  C* A = Mi + LL;
  C* B = A + L * L * P;
  for (int m = threadIdx.x; m < P; m += blockDim.x) {
    double s, c;
    sincospi(-2.0 * m / P, &s, &c);
    W[m].x = (T)c;
    W[m].y = (T)s;
  }
  for (int64_t e = blockIdx.x; e < n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < LL; i += blockDim.x) Mi[i] = M[e * LL + i];
    __syncthreads();
    for (int o = threadIdx.x; o < L * L * P; o += blockDim.x) {
      const int ab = o / P, k2 = o % P;
      C acc = czero<C>();
#pragma unroll
      for (int c = 0; c < L; c++) cfma(acc, Mi[ab * L + c], W[(k2 * c) % P]);
      A[o] = acc;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < L * P * P; o += blockDim.x) {
      const int a = o / (P * P), k1 = (o / P) % P, k2 = o % P;
      C acc = czero<C>();
#pragma unroll
      for (int b = 0; b < L; b++) cfma(acc, A[(a * L + b) * P + k2], W[(k1 * b) % P]);
      B[o] = acc;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < PP; o += blockDim.x) {
      const int k0 = o / (P * P), k12 = o % (P * P);
      C acc = czero<C>();
#pragma unroll
      for (int a = 0; a < L; a++) cfma(acc, B[a * P * P + k12], W[(k0 * a) % P]);
      F[e * PP + o] = acc;
    }
  }
}

// L[a,b,c] += (1/PP) sum_k J[k] conj(w)^(k0 a + k1 b + k2 c), a,b,c < L
// (circulant.hpp:109-118: unnormalised backward DFT, gather at itilda, /PP)
template <typename T, int L>
__global__ void k_f2l(int64_t n, const typename cpx_t<T>::type* __restrict__ J,
                      typename cpx_t<T>::type* __restrict__ Lx) {
  typedef typename cpx_t<T>::type C;
  constexpr int P = 2 * L - 1, LL = L * L * L, PP = P * P * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* W = reinterpret_cast<C*>(smem_raw);
  C* Ji = W + P;
  C* Cb = Ji + PP;
  C* D = Cb + L * P * P;
  for (int m = threadIdx.x; m < P; m += blockDim.x) {
    double s, c;
    sincospi(2.0 * m / P, &s, &c);
    W[m].x = (T)c;
    W[m].y = (T)s;
  }
  const T inv = T(1) / T(PP);
  for (int64_t e = blockIdx.x; e < n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < PP; i += blockDim.x) Ji[i] = J[e * PP + i];
    __syncthreads();
    for (int o = threadIdx.x; o < L * P * P; o += blockDim.x) {
      const int a = o / (P * P), k12 = o % (P * P);
      C acc = czero<C>();
#pragma unroll
      for (int k0 = 0; k0 < P; k0++) cfma(acc, Ji[k0 * P * P + k12], W[(k0 * a) % P]);
      Cb[o] = acc;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < L * L * P; o += blockDim.x) {
      const int a = o / (L * P), b = (o / P) % L, k2 = o % P;
      C acc = czero<C>();
#pragma unroll
      for (int k1 = 0; k1 < P; k1++) cfma(acc, Cb[(a * P + k1) * P + k2], W[(k1 * b) % P]);
      D[o] = acc;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < LL; o += blockDim.x) {
      const int ab = o / L, c = o % L;
      C acc = czero<C>();
#pragma unroll
      for (int k2 = 0; k2 < P; k2++) cfma(acc, D[ab * P + k2], W[(k2 * c) % P]);
      C v = Lx[e * LL + o];
      v.x += acc.x * inv;
      v.y += acc.y * inv;
      Lx[e * LL + o] = v;
    }
  }
}

// -------------------------------------------------------------------- M2L --
// One CTA per target slot of a cone batch (M2L.hpp:115-157, target-
// stationary):  J_t[i] = sum_{(s, u, h) in list(t)} u[perm_h[i]] * F_s[i]
template <typename T, int L, int NT>
__global__ void __launch_bounds__(NT) k_m2l(DevPlan P, int64_t t0, int64_t t1, int64_t f0, int64_t f1,
                                            const typename cpx_t<T>::type* __restrict__ F,
                                            const typename cpx_t<T>::type* __restrict__ tables,
                                            typename cpx_t<T>::type* __restrict__ J) {
  typedef typename cpx_t<T>::type C;
  constexpr int PD = 2 * L - 1, PP = PD * PD * PD, K = (PP + NT - 1) / NT;
  for (int64_t t = t0 + blockIdx.x; t < t1; t += gridDim.x) {
    C acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = czero<C>();
    const int64_t eb = P.m2l_ptr[t], ee = P.m2l_ptr[t + 1];
    for (int64_t e = eb; e < ee; e++) {
      const int64_t src = P.m2l_src[e];
      const uint32_t tb = P.m2l_tab[e];
      if (src < f0 || src >= f1) {  // entry outside this cone batch: a plan bug
        if (threadIdx.x == 0) atomicExch(P.err, 1);
        continue;
      }
      const C* Fs = F + (src - f0) * PP;
      const C* U = tables + (int64_t)(tb >> 6) * PP;
      const uint16_t* pm = P.perm + (int64_t)(tb & 63) * PP;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const int i = threadIdx.x + k * NT;
        if (i < PP) cfma(acc[k], U[pm[i]], Fs[i]);
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int i = threadIdx.x + k * NT;
      if (i < PP) J[(t - t0) * PP + i] = acc[k];
    }
  }
}

// -------------------------------------------------------------------- L2P --
// One CTA (4 warps) per target leaf at a precomputed level
// (dwnpass.hpp:39-47): HF (phfL2P, L2P.hpp:122-142)
//   p_j = sum_d exp(i k d.(x_j - c)) sum_l Z(j, l) sig2_d[l] L_d[l]
// LF (plfL2P :165-173): p_j = sum_l Z(j, l) L[l].  Writes p_far.
template <typename T, int L>
__global__ void __launch_bounds__(128) k_l2p(DevPlan P, const int32_t* __restrict__ leaves, int nleaves,
                                             const typename cpx_t<T>::type* __restrict__ sig2,
                                             const typename cpx_t<T>::type* __restrict__ Lx,
                                             double2* __restrict__ pfar) {
  typedef typename cpx_t<T>::type C;
  constexpr int LL = L * L * L;
  constexpr int NPB = 64;
  __shared__ T Bs[NPB][3][L];
  __shared__ C buf[4][LL];
  __shared__ double2 pacc[4][NPB];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int li = blockIdx.x; li < nleaves; li += gridDim.x) {
    const int c = leaves[li];
    const int n = P.T_nprt[c], f = P.T_first[c];
    const double4 ct = P.T_ctr[c];
    const int lv = P.T_lvl[c];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const int64_t sb = P.T_cptr[c], se = P.T_cptr[c + 1];
    const double* dirs = P.dirs + P.dir_off[h] * 3;
    const C* s2 = sig2 + P.sig_off[h];
    for (int p0 = 0; p0 < n; p0 += NPB) {
      const int np = min(NPB, n - p0);
      __syncthreads();
      for (int o = threadIdx.x; o < 3 * np; o += blockDim.x) {
        const int p = o / 3, k = o % 3;
        const double x = P.T_pos[3 * (int64_t)(f + p0 + p) + k] - (&ct.x)[k];
        T b[L];
        lagrange_all<L, T>((T)x, (T)ct.w, b);
#pragma unroll
        for (int l = 0; l < L; l++) Bs[p][k][l] = b[l];
      }
      for (int o = threadIdx.x; o < 4 * NPB; o += blockDim.x) pacc[o / NPB][o % NPB] = make_double2(0., 0.);
      __syncthreads();
      for (int64_t j = sb + warp; j < se; j += 4) {
        const int slot = P.T_cslot[j], d = P.T_cdir[j];
        const C* Ls = Lx + (int64_t)slot * LL;
        for (int l = lane; l < LL; l += 32) buf[warp][l] = hf ? cmul(s2[(int64_t)d * LL + l], Ls[l]) : Ls[l];
        __syncwarp();
        for (int p = lane; p < np; p += 32) {
          C acc = czero<C>();
          for (int l = 0; l < LL; l++) {
            const int i0 = l / (L * L), i1 = (l / L) % L, i2 = l % L;
            rfma(acc, Bs[p][0][i0] * Bs[p][1][i1] * Bs[p][2][i2], buf[warp][l]);
          }
          double2 a = make_double2((double)acc.x, (double)acc.y);
          if (hf) {
            const double* x = P.T_pos + 3 * (int64_t)(f + p0 + p);
            const double* dv = dirs + 3 * d;
            double dp = 0.;
            for (int k = 0; k < 3; k++) dp += dv[k] * (x[k] - (&ct.x)[k]);
            a = cmul(a, expi64<double2>(P.kappa * dp));
          }
          pacc[warp][p].x += a.x;
          pacc[warp][p].y += a.y;
        }
        __syncwarp();
      }
      __syncthreads();
      for (int p = threadIdx.x; p < np; p += blockDim.x) {
        double2 s = pacc[0][p];
        for (int w = 1; w < 4; w++) {
          s.x += pacc[w][p].x;
          s.y += pacc[w][p].y;
        }
        pfar[f + p0 + p] = s;
      }
    }
  }
}

// -------------------------------------------------------------------- P2P --
// Near field (P2P.hpp:43-79) on whole cells, target-stationary: one warp per
// chunk of <= 32 target particles of one leaf.  Lanes split into groups of
// tp >= nt lanes (one target each); groups take interleaved sources and are
// reduced by shuffles.  Pairs with r^2 < 1e-16 contribute nothing.  Writes
// p_near.  FP64 throughout.
__global__ void __launch_bounds__(256) k_p2p_fp64(DevPlan P, int64_t nchunk, const int32_t* __restrict__ tfirst,
                                                  const int32_t* __restrict__ tn, const int64_t* __restrict__ ptr,
                                                  const int32_t* __restrict__ sfirst, const int32_t* __restrict__ sn,
                                                  const double2* __restrict__ q, double2* __restrict__ pnear) {
  const int lane = threadIdx.x & 31;
  const double pi4m1 = 1. / (4. * 3.14159265358979323846);
  for (int64_t ch = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); ch < nchunk;
       ch += (int64_t)gridDim.x * (blockDim.x >> 5)) {
    const int f = tfirst[ch], nt = tn[ch];
    int tp = 1;
    while (tp < nt) tp <<= 1;
    const int groups = 32 / tp;
    const int mt = lane & (tp - 1), g = lane / tp;
    const int ti = f + min(mt, nt - 1);
    const double x0 = P.T_pos[3 * (int64_t)ti], x1 = P.T_pos[3 * (int64_t)ti + 1], x2 = P.T_pos[3 * (int64_t)ti + 2];
    double pr = 0., pim = 0.;
    const int64_t rb = ptr[ch], re = ptr[ch + 1];
    for (int64_t r = rb; r < re; r++) {
      const int sf = sfirst[r], ns = sn[r];
      for (int j = g; j < ns; j += groups) {
        const int64_t sj = sf + j;
        const double y0 = P.S_pos[3 * sj], y1 = P.S_pos[3 * sj + 1], y2 = P.S_pos[3 * sj + 2];
        const double2 qq = q[sj];
        const double dx = x0 - y0, dy = x1 - y1, dz = x2 - y2;
        const double R = dx * dx + dy * dy + dz * dz;
        double K = rsqrt(R);
        if (R < 1.e-16) K = 0.;
        const double rr = K * R * P.kappa;
        K *= pi4m1;
        double s, c;
        sincos(rr, &s, &c);
        c *= K;
        s *= K;
        pr += c * qq.x - s * qq.y;
        pim += c * qq.y + s * qq.x;
      }
    }
    for (int off = tp; off < 32; off <<= 1) {
      pr += __shfl_xor_sync(0xffffffffu, pr, off);
      pim += __shfl_xor_sync(0xffffffffu, pim, off);
    }
    if (g == 0 && mt < nt) pnear[f + mt] = make_double2(pr, pim);
  }
}

// ------------------------------------------------------------ direct sum --
// FP64 direct sum at sampled targets (CheckFULL arithmetic,
// interface.hpp:178-221): one warp per target, lanes over sources.
__global__ void k_direct(int64_t ns, const double* __restrict__ spos, const int32_t* __restrict__ sperm,
                         const double2* __restrict__ qin, int64_t nt, const double* __restrict__ tpos,
                         double kappa, double2* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const double pi4m1 = 1. / (4. * 3.14159265358979323846);
  for (int64_t t = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); t < nt;
       t += (int64_t)gridDim.x * (blockDim.x >> 5)) {
    const double x0 = tpos[3 * t], x1 = tpos[3 * t + 1], x2 = tpos[3 * t + 2];
    double pr = 0., pim = 0.;
    for (int64_t j = lane; j < ns; j += 32) {
      const double dx = x0 - spos[3 * j], dy = x1 - spos[3 * j + 1], dz = x2 - spos[3 * j + 2];
      const double R = dx * dx + dy * dy + dz * dz;
      double K = 1. / sqrt(R);
      if (R < 1.e-16) K = 0.;
      const double rr = K * R * kappa;
      K *= pi4m1;
      double s, c;
      sincos(rr, &s, &c);
      const double2 qq = qin[sperm[j]];
      pr += c * K * qq.x - s * K * qq.y;
      pim += c * K * qq.y + s * K * qq.x;
    }
    for (int off = 16; off; off >>= 1) {
      pr += __shfl_xor_sync(0xffffffffu, pr, off);
      pim += __shfl_xor_sync(0xffffffffu, pim, off);
    }
    if (lane == 0) out[t] = make_double2(pr, pim);
  }
}

// ---------------------------------------------------------------- launch --
namespace {
int grid_for(int64_t n, int per_block, int cap = 148 * 64) {
  int64_t g = (n + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}
}  // namespace

template <typename T, int L>
struct Launch {
  typedef typename cpx_t<T>::type C;
  static constexpr int P = 2 * L - 1, LL = L * L * L, PP = P * P * P;
  static constexpr int NT = PP > 1024 ? 256 : 128;
  static size_t smem_m2f() { return sizeof(C) * (P + LL + L * L * P + L * P * P); }
  static size_t smem_f2l() { return sizeof(C) * (P + PP + L * P * P + L * L * P); }
  static cudaError_t setup() {
    cudaError_t e = cudaFuncSetAttribute(k_m2f<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_m2f());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_f2l<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_f2l());
  }
  static void p2m(const DevPlan& dp, const int32_t* leaves, int n, const void* q, const void* sig2, void* M,
                  cudaStream_t s) {
    if (n) k_p2m<T, L><<<grid_for(n, 1), 128, 0, s>>>(dp, leaves, n, (const C*)q, (const C*)sig2, (C*)M);
  }
  static void m2m(const DevPlan& dp, int64_t s0, int64_t s1, const void* sig, const void* sig2, void* M,
                  cudaStream_t s) {
    constexpr int NW = XferCfg<T, L>::NW;
    if (s1 > s0) k_m2m<T, L><<<grid_for(s1 - s0, NW), 32 * NW, 0, s>>>(dp, s0, s1, (const C*)sig, (const C*)sig2, (C*)M);
  }
  static void l2l(const DevPlan& dp, int64_t s0, int64_t s1, const void* sig, const void* sig2, void* Lx,
                  cudaStream_t s) {
    constexpr int NW = XferCfg<T, L>::NW;
    if (s1 > s0) k_l2l<T, L><<<grid_for(s1 - s0, NW), 32 * NW, 0, s>>>(dp, s0, s1, (const C*)sig, (const C*)sig2, (C*)Lx);
  }
  static void m2f(int64_t n, const void* M, void* F, cudaStream_t s) {
    if (n) k_m2f<T, L><<<grid_for(n, 1), 128, smem_m2f(), s>>>(n, (const C*)M, (C*)F);
  }
  static void f2l(int64_t n, const void* J, void* Lx, cudaStream_t s) {
    if (n) k_f2l<T, L><<<grid_for(n, 1), 128, smem_f2l(), s>>>(n, (const C*)J, (C*)Lx);
  }
  static void m2l(const DevPlan& dp, int64_t t0, int64_t t1, int64_t f0, int64_t f1, const void* F,
                  const void* tables, void* J, cudaStream_t s) {
    if (t1 > t0)
      k_m2l<T, L, NT><<<grid_for(t1 - t0, 1), NT, 0, s>>>(dp, t0, t1, f0, f1, (const C*)F, (const C*)tables, (C*)J);
  }
  static void l2p(const DevPlan& dp, const int32_t* leaves, int n, const void* sig2, const void* Lx, double2* pfar,
                  cudaStream_t s) {
    if (n) k_l2p<T, L><<<grid_for(n, 1), 128, 0, s>>>(dp, leaves, n, (const C*)sig2, (const C*)Lx, pfar);
  }
};

template <typename T>
const OpTable* op_table_for(int L);

#define DFB_OPS(T, L)                                                                                     \
  {                                                                                                       \
    Launch<T, L>::setup, Launch<T, L>::p2m, Launch<T, L>::m2m, Launch<T, L>::l2l, Launch<T, L>::m2f,       \
        Launch<T, L>::f2l, Launch<T, L>::m2l, Launch<T, L>::l2p                                           \
  }

template <>
const OpTable* op_table_for<double>(int L) {
  static const OpTable t[9] = {{},
                               {},
                               DFB_OPS(double, 2),
                               DFB_OPS(double, 3),
                               DFB_OPS(double, 4),
                               DFB_OPS(double, 5),
                               DFB_OPS(double, 6),
                               DFB_OPS(double, 7),
                               DFB_OPS(double, 8)};
  return (L >= 2 && L <= 8) ? &t[L] : nullptr;
}

template <>
const OpTable* op_table_for<float>(int L) {
  static const OpTable t[9] = {{},
                               {},
                               DFB_OPS(float, 2),
                               DFB_OPS(float, 3),
                               DFB_OPS(float, 4),
                               DFB_OPS(float, 5),
                               DFB_OPS(float, 6),
                               DFB_OPS(float, 7),
                               DFB_OPS(float, 8)};
  return (L >= 2 && L <= 8) ? &t[L] : nullptr;
}

const OpTable* op_table(int L, bool fp64) { return fp64 ? op_table_for<double>(L) : op_table_for<float>(L); }

void launch_gather(bool fp64, const double2* qin, const int32_t* perm, void* q, int64_t n, int64_t sin_, int64_t sq,
                   int nrhs, cudaStream_t s) {
  const int g = (int)((n + 255) / 256);
  if (fp64)
    k_gather<double><<<g, 256, 0, s>>>(qin, perm, (double2*)q, n, sin_, sq, nrhs);
  else
    k_gather<float><<<g, 256, 0, s>>>(qin, perm, (float2*)q, n, sin_, sq, nrhs);
}

void launch_scatter(const double2* pnear, const double2* pfar, const int32_t* perm, double2* out, int64_t n,
                    cudaStream_t s) {
  k_scatter<<<(int)((n + 255) / 256), 256, 0, s>>>(pnear, pfar, perm, out, n);
}

void launch_p2p_fp64(const DevPlan& dp, int64_t nchunk, const int32_t* tfirst, const int32_t* tn, const int64_t* ptr,
                     const int32_t* sfirst, const int32_t* sn, const double2* q, double2* pnear, cudaStream_t s) {
  if (nchunk) k_p2p_fp64<<<grid_for(nchunk, 8, 148 * 32), 256, 0, s>>>(dp, nchunk, tfirst, tn, ptr, sfirst, sn, q, pnear);
}

void launch_direct(int64_t ns, const double* spos, const int32_t* sperm, const double2* qin, int64_t nt,
                   const double* tpos, double kappa, double2* out, cudaStream_t s) {
  if (nt) k_direct<<<grid_for(nt, 8, 148 * 16), 256, 0, s>>>(ns, spos, sperm, qin, nt, tpos, kappa, out);
}

}  // namespace dfb
