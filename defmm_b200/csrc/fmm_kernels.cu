// Matvec kernels.  One template per phase, instantiated per precision (T)
// and interpolation order (L).  See kernels.cuh for the memory layout.
#include "kernels.cuh"
#include "device_math.cuh"
#include "fmm_kernels.h"
#include "ptx.cuh"

#include <algorithm>
#include <mutex>
#include <set>
#include <type_traits>
#include <utility>
#include <vector>

namespace dfb {

// --------------------------------------------------------- constant tables --
// Per order L = 2..8: the four L x L interpolation matrices (m2m[0], m2m[1],
// l2l[0], l2l[1]; A(k, p) at k + p L) and the twiddles exp(-2 pi i m / P),
// P = 2L - 1.  Every use sits in a fully unrolled loop, so the operands are
// immediate constant-bank addresses rather than shared-memory loads.
constexpr int kMinOrder = 2, kMaxOrder = 8;
__host__ __device__ constexpr int mat_off(int L) {
  int s = 0;
  for (int l = kMinOrder; l < L; l++) s += 4 * l * l;
  return s;
}
__host__ __device__ constexpr int tw_off(int L) {
  int s = 0;
  for (int l = kMinOrder; l < L; l++) s += 2 * l - 1;
  return s;
}
__constant__ double c_mat64[mat_off(kMaxOrder + 1)];
__constant__ float c_mat32[mat_off(kMaxOrder + 1)];
__constant__ double c_tw64[2 * tw_off(kMaxOrder + 1)];
__constant__ float c_tw32[2 * tw_off(kMaxOrder + 1)];

template <typename T>
__device__ __forceinline__ T cmat(int i);
template <>
__device__ __forceinline__ double cmat<double>(int i) {
  return c_mat64[i];
}
template <>
__device__ __forceinline__ float cmat<float>(int i) {
  return c_mat32[i];
}
// twiddle exp(-2 pi i m / P) of order L, m in [0, P)
template <typename T, int L>
__device__ __forceinline__ typename cpx_t<T>::type ctw(int m) {
  typename cpx_t<T>::type r;
  if constexpr (sizeof(T) == 8) {
    r.x = c_tw64[2 * (tw_off(L) + m)];
    r.y = c_tw64[2 * (tw_off(L) + m) + 1];
  } else {
    r.x = c_tw32[2 * (tw_off(L) + m)];
    r.y = c_tw32[2 * (tw_off(L) + m) + 1];
  }
  return r;
}
// acc += v * conj(w)
template <typename C>
__device__ __forceinline__ void cfmac(C& acc, C v, C w) {
  acc.x = fma(v.x, w.x, acc.x);
  acc.x = fma(v.y, w.y, acc.x);
  acc.y = fma(v.y, w.x, acc.y);
  acc.y = fma(-v.x, w.y, acc.y);
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
// HF leaf (phfP2M, P2M.hpp:114-131), per effective direction d:
//   M_d[l] = conj(sig2_d[l]) * sum_j Z(l, j) exp(-i k d.(y_j - c)) q_j
// LF leaf (plfP2M, P2M.hpp:134-136): M[l] = sum_j Z(l, j) q_j,
// with Z(l, j) = prod_k S_{I_k(l)}(y_jk - c_k) the leaf's interpolation matrix
// (mapOnTrees.hpp:37-83).
//
// Per leaf this is the small GEMM  M[l][s] = sum_j Z[j][l] W[j][s],
// W[j][s] = q_j exp(-i k d_s.(y_j - c)).  One CTA per leaf, in chunks of NPB
// points: Z[j][l] is built once per chunk in shared memory (point-major, l
// padded to LLP = 32 R); each warp takes S of the leaf's slots at a time,
// writes their W column block, and every lane accumulates an R x S register
// tile (expansion entries R lane .. R lane + R - 1, all S slots) over the
// chunk's points: per point one R-wide load of Z and S broadcast loads of W
// feed 2 R S FMAs.
template <typename T, int L>
struct P2MCfg {
  static constexpr int LL = L * L * L;
  static constexpr int R = L >= 5 ? 4 * ((LL + 127) / 128) : (LL + 31) / 32;  // entries per lane
  static constexpr int LLP = 32 * R;
  static constexpr int S0 = (sizeof(T) == 4 ? 32 : 16) / R;
  static constexpr int S = S0 < 1 ? 1 : (S0 > (sizeof(T) == 4 ? 8 : 4) ? (sizeof(T) == 4 ? 8 : 4) : S0);
  static constexpr int NPB0 = 65536 / (LLP * (int)sizeof(T));
  static constexpr int NPB = NPB0 > 64 ? 64 : NPB0;  // points per chunk
  typedef typename cpx_t<T>::type C;
  // shared memory: Z, point offsets, basis values, W blocks of 4 warps,
  // (with R > 1 right-hand sides) phase blocks of 4 warps, charges (R per point)
  static constexpr size_t smem(int R = 1) {
    return sizeof(T) * (size_t)NPB * LLP + sizeof(double) * NPB * 3 + sizeof(T) * NPB * 3 * L +
           sizeof(C) * 4 * NPB * S * (R > 1 ? 2 : 1) + sizeof(C) * (size_t)NPB * R;
  }
};

template <typename T, int L, int SS>
__device__ __forceinline__ void p2m_group(const DevPlan& P, int64_t j0, int ns, bool hf, bool first, int np,
                                          const T* __restrict__ Zs, const double* __restrict__ yc,
                                          const typename cpx_t<T>::type* __restrict__ qs,
                                          typename cpx_t<T>::type* __restrict__ Ws,
                                          typename cpx_t<T>::type* __restrict__ Es, const double* dirs,
                                          const typename cpx_t<T>::type* __restrict__ s2,
                                          typename cpx_t<T>::type* __restrict__ M, int R, int lane) {
  typedef typename cpx_t<T>::type C;
  typedef P2MCfg<T, L> G;
  constexpr int RE = G::R, LLP = G::LLP, LL = G::LL;
  __syncwarp();
  // phases exp(-i k d_s.(y_j - c)) of the group's slots, shared by the
  // right-hand sides (with one right-hand side the charge is folded in here)
  for (int idx = lane; idx < np * SS; idx += 32) {
    const int j = idx / SS, s = idx % SS;
    C w;
    if (s >= ns) {
      w = czero<C>();
    } else if (hf) {
      const double* dv = dirs + 3 * P.S_cdir[j0 + s];
      double dp = 0.;
      for (int k = 0; k < 3; k++) dp += dv[k] * yc[3 * j + k];
      w = expi<C>(-P.kappa * dp);
    } else {
      w.x = T(1);
      w.y = T(0);
    }
    if (R == 1)
      Ws[j * SS + s] = cmul(w, qs[j]);
    else
      Es[j * SS + s] = w;
  }
  for (int r = 0; r < R; r++) {
    __syncwarp();
    if (R > 1) {
      for (int idx = lane; idx < np * SS; idx += 32) {
        const int j = idx / SS;
        Ws[idx] = cmul(Es[idx], qs[j * R + r]);
      }
      __syncwarp();
    }
    C acc[RE][SS];
#pragma unroll
    for (int e = 0; e < RE; e++)
#pragma unroll
      for (int s = 0; s < SS; s++) acc[e][s] = czero<C>();
    const T* zl = Zs + lane * RE;
    for (int j = 0; j < np; j++) {
      T z[RE];
      C w[SS];
#pragma unroll
      for (int e = 0; e < RE; e++) z[e] = zl[j * LLP + e];
#pragma unroll
      for (int s = 0; s < SS; s++) w[s] = Ws[j * SS + s];
#pragma unroll
      for (int e = 0; e < RE; e++)
#pragma unroll
        for (int s = 0; s < SS; s++) rfma(acc[e][s], z[e], w[s]);
    }
#pragma unroll
    for (int s = 0; s < SS; s++) {
      if (s < ns) {
        const int slot = P.S_cslot[j0 + s], d = P.S_cdir[j0 + s];
#pragma unroll
        for (int e = 0; e < RE; e++) {
          const int l = lane * RE + e;
          if (l < LL) {
            const C a = hf ? cmulc(s2[(int64_t)d * LL + l], acc[e][s]) : acc[e][s];
            C* out = M + ((int64_t)slot * R + r) * LL + l;
            if (first) {
              *out = a;
            } else {
              C o = *out;
              o.x += a.x;
              o.y += a.y;
              *out = o;
            }
          }
        }
      }
    }
  }
}

// M: base of the expansions written here (slot s, right-hand side r at
// M + (s R + r) LL); q: tree-order charges, R per particle (q[j R + r]);
// only the leaf slots with a direction in [d0, d1) are computed.
template <typename T, int L>
__global__ void __launch_bounds__(128) k_p2m(DevPlan P, const int32_t* __restrict__ leaves, int nleaves,
                                             const typename cpx_t<T>::type* __restrict__ q,
                                             const typename cpx_t<T>::type* __restrict__ sig2,
                                             typename cpx_t<T>::type* __restrict__ M, int R, int d0, int d1) {
  typedef typename cpx_t<T>::type C;
  typedef P2MCfg<T, L> G;
  constexpr int LL = G::LL, LLP = G::LLP, NPB = G::NPB, S = G::S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Zs = reinterpret_cast<T*>(smem_raw);
  double* yc = reinterpret_cast<double*>(Zs + (size_t)NPB * LLP);
  T* Bs = reinterpret_cast<T*>(yc + NPB * 3);
  C* Wall = reinterpret_cast<C*>(Bs + NPB * 3 * L);
  C* Eall = Wall + 4 * NPB * S;
  C* qs = Eall + (R > 1 ? 4 * NPB * S : 0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* Ws = Wall + warp * NPB * S;
  C* Es = Eall + warp * NPB * S;
  for (int li = blockIdx.x; li < nleaves; li += gridDim.x) {
    const int c = leaves[li];
    const int n = P.S_nprt[c], f = P.S_first[c];
    const double4 ct = P.S_ctr[c];
    const int lv = P.S_lvl[c];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    int64_t sb, se;
    dir_range(P.S_cptr, P.S_cdir, c, d0, d1, &sb, &se);
    const int nslots = (int)(se - sb);
    if (nslots == 0) continue;
    const double* dirs = P.dirs + P.dir_off[h] * 3;
    const C* s2 = sig2 + P.sig_off[h];
    for (int p0 = 0; p0 < n; p0 += NPB) {
      const int np = min(NPB, n - p0);
      __syncthreads();  // the previous chunk's Z, W are no longer read
      for (int o = threadIdx.x; o < 3 * np; o += blockDim.x) {
        const int p = o / 3, k = o % 3;
        const double x = P.S_pos[3 * (int64_t)(f + p0 + p) + k] - (&ct.x)[k];
        yc[o] = x;
        T b[L];
        lagrange_all<L, T>((T)x, (T)ct.w, b);
#pragma unroll
        for (int l = 0; l < L; l++) Bs[(p * 3 + k) * L + l] = b[l];
      }
      for (int p = threadIdx.x; p < np * R; p += blockDim.x) qs[p] = q[(int64_t)(f + p0) * R + p];
      __syncthreads();
      for (int o = threadIdx.x; o < np * LLP; o += blockDim.x) {
        const int p = o / LLP, l = o % LLP;
        T z = 0;
        if (l < LL) {
          const int i0 = l / (L * L), i1 = (l / L) % L, i2 = l % L;
          z = Bs[(p * 3 + 0) * L + i0] * Bs[(p * 3 + 1) * L + i1] * Bs[(p * 3 + 2) * L + i2];
        }
        Zs[o] = z;
      }
      __syncthreads();
      for (int g0 = warp * S; g0 < nslots; g0 += 4 * S) {
        const int ns = min(S, nslots - g0);
        if (ns == 1)
          p2m_group<T, L, 1>(P, sb + g0, 1, hf, p0 == 0, np, Zs, yc, qs, Ws, Es, dirs, s2, M, R, lane);
        else
          p2m_group<T, L, S>(P, sb + g0, ns, hf, p0 == 0, np, Zs, yc, qs, Ws, Es, dirs, s2, M, R, lane);
      }
    }
  }
}

// ------------------------------------------------ separable 3-D transfer --
// out[a,b,c] = sum A_s0(a,a') A_s1(b,b') A_s2(c,c') in[a',b',c'] computed in
// three axis passes (axis 2, 1, 0 as interpolation.hpp:311-361); A(k, p) is
// matrix 2*ROLE + s of the order's constant table (ROLE 0: M2M, 1: L2L).
// One warp per transfer; lane ln owns line(s) ln, ln + 32 of each pass:
//   axis 2 on (a, b) lines: input in registers (v), output to buf
//   axis 1 on (a, c) lines: in place in buf (a lane's line is its own)
//   axis 0 on (b, c) lines: from buf to registers (res)
// The branch on each s is warp-uniform and keeps the matrix indices
// compile-time constants.
template <typename T, int L, int ROLE>
struct Sep {
  typedef typename cpx_t<T>::type C;
  static constexpr int NLN = (L * L + 31) / 32;  // lines per lane
  template <int MI>
  __device__ static __forceinline__ void line(const C (&v)[L], C (&o)[L]) {
    constexpr int B = mat_off(L) + MI * L * L;
#pragma unroll
    for (int k = 0; k < L; k++) {
      C acc = czero<C>();
#pragma unroll
      for (int p = 0; p < L; p++) rfma(acc, cmat<T>(B + k + p * L), v[p]);
      o[k] = acc;
    }
  }
  __device__ static __forceinline__ void apply(int s, const C (&v)[L], C (&o)[L]) {
    if (s)
      line<2 * ROLE + 1>(v, o);
    else
      line<2 * ROLE>(v, o);
  }
  // The same transfer with the passes in the order axis 0, 1, 2: the input
  // lines run along axis 0 (v[q][p] = in[p, b, c] for line (b, c) = ln, so a
  // warp reads an expansion with unit stride across lanes), res holds lines
  // (a, b) = ln along axis 2 (res[q][k] = out[a, b, k]).
  __device__ static __forceinline__ void run_a0(int sg0, int sg1, int sg2, const C (&v)[NLN][L], C* buf,
                                                C (&res)[NLN][L], int lane) {
#pragma unroll
    for (int q = 0; q < NLN; q++) {  // axis 0: lines (b, c)
      const int ln = lane + 32 * q;
      if (ln < L * L) {
        C o[L];
        apply(sg0, v[q], o);
#pragma unroll
        for (int k = 0; k < L; k++) buf[k * L * L + ln] = o[k];
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NLN; q++) {  // axis 1: lines (a, c), in place
      const int ln = lane + 32 * q;
      if (ln < L * L) {
        const int a = ln / L, c = ln % L;
        C w[L], o[L];
#pragma unroll
        for (int p = 0; p < L; p++) w[p] = buf[(a * L + p) * L + c];
        apply(sg1, w, o);
#pragma unroll
        for (int k = 0; k < L; k++) buf[(a * L + k) * L + c] = o[k];
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NLN; q++) {  // axis 2: lines (a, b)
      const int ln = lane + 32 * q;
      if (ln < L * L) {
        C w[L];
#pragma unroll
        for (int p = 0; p < L; p++) w[p] = buf[ln * L + p];
        apply(sg2, w, res[q]);
      }
    }
    __syncwarp();
  }
  __device__ static __forceinline__ void run(int sg0, int sg1, int sg2, const C (&v)[NLN][L], C* buf,
                                             C (&res)[NLN][L], int lane) {
#pragma unroll
    for (int q = 0; q < NLN; q++) {  // axis 2: lines (a, b)
      const int ln = lane + 32 * q;
      if (ln < L * L) {
        C o[L];
        apply(sg2, v[q], o);
#pragma unroll
        for (int k = 0; k < L; k++) buf[ln * L + k] = o[k];
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NLN; q++) {  // axis 1: lines (a, c), in place
      const int ln = lane + 32 * q;
      if (ln < L * L) {
        const int a = ln / L, c = ln % L;
        C w[L], o[L];
#pragma unroll
        for (int p = 0; p < L; p++) w[p] = buf[(a * L + p) * L + c];
        apply(sg1, w, o);
#pragma unroll
        for (int k = 0; k < L; k++) buf[(a * L + k) * L + c] = o[k];
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NLN; q++) {  // axis 0: lines (b, c)
      const int ln = lane + 32 * q;
      if (ln < L * L) {
        C w[L];
#pragma unroll
        for (int p = 0; p < L; p++) w[p] = buf[p * L * L + ln];
        apply(sg0, w, res[q]);
      }
    }
    __syncwarp();
  }
};

// -------------------------------------------------------------------- M2M --
// One warp per parent slot with children (upwpass.hpp:49-60):
//   HF parent, direction d (hfM2Mblock M2M.hpp:76-105 / lf2hfM2M :108-124):
//     M_d = conj(sig2_d) o sum_c exp(-i k d.v_c) A_{v_c}(sig_d o M_c)
//   LF parent (lfM2M :35-41): M = sum_c A_{v_c}(M_c);   v_c = ctr_c - ctr_parent
// A lane reads its (b, c) lines (along axis 0) of each child's expansion
// straight into registers, lanes at unit stride (the next child's are
// prefetched during the current transfer); the transfer runs axis 0 first.
// Lane e holds child e's slot, octant and plane-wave phase, computed once
// per parent slot.  With R right-hand sides a warp takes one parent slot and
// runs its transfers for every right-hand side in turn; the parent's
// expansions live at Mp + (slot R + r) LL, the children's at
// Mc0 + (slot R + r) LL (both bases may be the same array).
constexpr int kXferWarps = 4;  // warps (transfers in flight) per CTA

template <typename T, int L>
__global__ void __launch_bounds__(32 * kXferWarps, sizeof(T) == 4 ? (L <= 5 ? 6 : 3) : (L <= 5 ? 3 : 1)) k_m2m(DevPlan P, int64_t s0, int64_t s1,
                                                         const typename cpx_t<T>::type* __restrict__ sig,
                                                         const typename cpx_t<T>::type* __restrict__ sig2,
                                                         typename cpx_t<T>::type* __restrict__ Mp,
                                                         const typename cpx_t<T>::type* __restrict__ Mc0, int R) {
  typedef typename cpx_t<T>::type C;
  typedef Sep<T, L, 0> S;
  constexpr int LL = L * L * L, NW = kXferWarps, NLN = S::NLN;
  __shared__ C sbuf[NW][LL];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t ps = s0 + blockIdx.x * NW + warp; ps < s1; ps += (int64_t)gridDim.x * NW) {
    const int64_t eb = P.m2m_ptr[ps], ee = P.m2m_ptr[ps + 1];
    if (eb == ee) continue;  // leaf slot: written by P2M
    const int pc = P.sS_cell[ps], d = P.sS_dir[ps];
    const int lv = P.S_lvl[pc];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const C* sg = sig + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
    const C* sg2 = sig2 + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
    // child e (<= 8) on lane e: its slot, the octant of its centre (bit k
    // set when v_k >= 0) and its phase exp(-i k d.v)
    const int nch = (int)(ee - eb);
    int my_cs = 0, my_oct = 0;
    C my_ph = czero<C>();
    if (lane < nch) {
      my_cs = P.m2m_child[eb + lane];
      const double4 pct = P.S_ctr[pc], ct = P.S_ctr[P.sS_cell[my_cs]];
      const double v0 = ct.x - pct.x, v1 = ct.y - pct.y, v2 = ct.z - pct.z;
      my_oct = (v0 < 0. ? 0 : 1) | (v1 < 0. ? 0 : 2) | (v2 < 0. ? 0 : 4);
      if (hf) {
        const double* dv = P.dirs + 3 * (P.dir_off[h] + d);
        my_ph = expi<C>(-P.kappa * (dv[0] * v0 + dv[1] * v1 + dv[2] * v2));
      }
    }
    // with one line per lane (L <= 5) the parent's signature line and the
    // next transfer's lines stay in registers; larger orders reload them
    constexpr bool REG = NLN == 1;
    C acc[NLN][L], sgr[REG ? NLN : 1][L];
#pragma unroll
    for (int q = 0; q < NLN; q++) {
      const int ln = lane + 32 * q;
#pragma unroll
      for (int k = 0; k < L; k++) {
        acc[q][k] = czero<C>();
        if (REG) sgr[0][k] = (hf && ln < L * L) ? sg[k * L * L + ln] : czero<C>();
      }
    }
    C nxt[REG ? NLN : 1][L];  // next transfer's (a, b) lines, prefetched
    if (REG) {
      const C* Mc = Mc0 + (int64_t)__shfl_sync(0xffffffffu, my_cs, 0) * R * LL;
#pragma unroll
      for (int k = 0; k < L; k++) nxt[0][k] = lane < L * L ? Mc[k * L * L + lane] : czero<C>();
    }
    // transfers in (right-hand side, child) order
    const int nit = nch * R;
    int e = 0, rr = 0;
    for (int it = 0; it < nit; it++) {
      const int oct = __shfl_sync(0xffffffffu, my_oct, e);
      C in[NLN][L];
      if (REG) {
#pragma unroll
        for (int k = 0; k < L; k++) in[0][k] = hf ? cmul(sgr[0][k], nxt[0][k]) : nxt[0][k];
        const int e1 = e + 1 < nch ? e + 1 : 0, r1 = e + 1 < nch ? rr : rr + 1;
        const int cs1 = __shfl_sync(0xffffffffu, my_cs, e1);
        if (it + 1 < nit) {
          const C* Mc = Mc0 + ((int64_t)cs1 * R + r1) * LL;
#pragma unroll
          for (int k = 0; k < L; k++)
            if (lane < L * L) nxt[0][k] = Mc[k * L * L + lane];
        }
      } else {
        const C* Mc = Mc0 + ((int64_t)__shfl_sync(0xffffffffu, my_cs, e) * R + rr) * LL;
#pragma unroll
        for (int q = 0; q < NLN; q++) {
          const int ln = lane + 32 * q;
#pragma unroll
          for (int k = 0; k < L; k++) {
            const C m = ln < L * L ? Mc[k * L * L + ln] : czero<C>();
            in[q][k] = (hf && ln < L * L) ? cmul(sg[k * L * L + ln], m) : m;
          }
        }
      }
      C res[NLN][L];
      S::run_a0(oct & 1, (oct >> 1) & 1, (oct >> 2) & 1, in, sbuf[warp], res, lane);
      if (hf) {
        C ph;
        ph.x = __shfl_sync(0xffffffffu, my_ph.x, e);
        ph.y = __shfl_sync(0xffffffffu, my_ph.y, e);
#pragma unroll
        for (int q = 0; q < NLN; q++)
#pragma unroll
          for (int k = 0; k < L; k++) cfma(acc[q][k], ph, res[q][k]);
      } else {
#pragma unroll
        for (int q = 0; q < NLN; q++)
#pragma unroll
          for (int k = 0; k < L; k++) {
            acc[q][k].x += res[q][k].x;
            acc[q][k].y += res[q][k].y;
          }
      }
      if (++e == nch) {  // the last child of right-hand side rr
#pragma unroll
        for (int q = 0; q < NLN; q++) {
          const int ln = lane + 32 * q;
#pragma unroll
          for (int k = 0; k < L; k++) {
            if (ln < L * L) {
              const int l = ln * L + k;
              Mp[(ps * R + rr) * LL + l] = hf ? cmulc(sg2[l], acc[q][k]) : acc[q][k];
            }
            acc[q][k] = czero<C>();
          }
        }
        e = 0;
        rr++;
      }
    }
  }
}

// -------------------------------------------------------------------- L2L --
// One warp per child slot with parents (dwnpass.hpp:49-58):
//   HF parent direction d (hfL2Lblock L2L.hpp:78-108 / hf2lfL2L :111-127):
//     L_c += sum_d exp(i k v.d) conj(sig_d) o B_v(sig2_d o L_d)
//   LF parent (lfL2L :35-41): L_c += B_v(L_p);   v = ctr_child - ctr_parent
// Lane e holds parent e's slot, direction and phase, computed once per child
// slot.  With R right-hand sides a warp takes one child slot and runs its
// transfers for every right-hand side in turn; children at
// Lc + (slot R + r) LL, parents at Lp0 + (slot R + r) LL.  Only
// parent slots in [p0, p1) contribute (a pass over part of the directions).
template <typename T, int L>
__global__ void __launch_bounds__(32 * kXferWarps, sizeof(T) == 4 ? (L <= 5 ? 6 : 3) : (L <= 5 ? 4 : 1)) k_l2l(DevPlan P, int64_t s0, int64_t s1,
                                                         const typename cpx_t<T>::type* __restrict__ sig,
                                                         const typename cpx_t<T>::type* __restrict__ sig2,
                                                         typename cpx_t<T>::type* __restrict__ Lc,
                                                         const typename cpx_t<T>::type* __restrict__ Lp0, int R,
                                                         int64_t p0, int64_t p1) {
  typedef typename cpx_t<T>::type C;
  typedef Sep<T, L, 1> S;
  constexpr int LL = L * L * L, NW = kXferWarps, NLN = S::NLN;
  __shared__ C sbuf[NW][LL];
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
    C acc[NLN][L];
#pragma unroll
    for (int q = 0; q < NLN; q++)
#pragma unroll
      for (int k = 0; k < L; k++) acc[q][k] = czero<C>();
    // parents' slots and directions fetched by lane (<= 6 per child slot),
    // only those in [p0, p1), compacted to the first lanes
    const int nall = (int)(ee - eb);
    int all_ps = 0, all_d = 0;
    if (lane < nall) {
      all_ps = P.l2l_parent[eb + lane];
      all_d = P.sT_dir[all_ps];
    }
    int my_ps = 0, my_d = 0, npa = 0;
    for (int e = 0; e < nall; e++) {  // warp-uniform: keep the parents in range, in order
      const int ps_e = __shfl_sync(0xffffffffu, all_ps, e);
      const int d_e = __shfl_sync(0xffffffffu, all_d, e);
      if (ps_e >= p0 && ps_e < p1) {
        if (lane == npa) {
          my_ps = ps_e;
          my_d = d_e;
        }
        npa++;
      }
    }
    if (npa == 0) continue;
    // parent e on lane e: its phase exp(i k v.d_e)
    C my_ph = czero<C>();
    if (hf && lane < npa) {
      const double* dv = P.dirs + 3 * (P.dir_off[h] + my_d);
      my_ph = expi<C>(P.kappa * (v[0] * dv[0] + v[1] * dv[1] + v[2] * dv[2]));
    }
    // with one line per lane (L <= 5) the next transfer's lines are
    // prefetched into registers; larger orders load them when used
    constexpr bool REG = NLN == 1;
    C nxt[REG ? NLN : 1][L];
    if (REG) {
      const C* Lp = Lp0 + (int64_t)__shfl_sync(0xffffffffu, my_ps, 0) * R * LL;
#pragma unroll
      for (int k = 0; k < L; k++) nxt[0][k] = lane < L * L ? Lp[lane * L + k] : czero<C>();
    }
    // transfers in (right-hand side, parent) order
    const int nit = npa * R;
    int e = 0, rr = 0;
    for (int it = 0; it < nit; it++) {
      const int d = __shfl_sync(0xffffffffu, my_d, e);
      const C* sg = sig + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
      const C* sgq = sig2 + P.sig_off[h] + (int64_t)(hf ? d : 0) * LL;
      C in[NLN][L];
      if (REG) {
#pragma unroll
        for (int k = 0; k < L; k++) in[0][k] = (hf && lane < L * L) ? cmul(sgq[lane * L + k], nxt[0][k]) : nxt[0][k];
        const int e1 = e + 1 < npa ? e + 1 : 0, r1 = e + 1 < npa ? rr : rr + 1;
        const int ps1 = __shfl_sync(0xffffffffu, my_ps, e1);
        if (it + 1 < nit) {
          const C* Lp = Lp0 + ((int64_t)ps1 * R + r1) * LL;
#pragma unroll
          for (int k = 0; k < L; k++)
            if (lane < L * L) nxt[0][k] = Lp[lane * L + k];
        }
      } else {
        const C* Lp = Lp0 + ((int64_t)__shfl_sync(0xffffffffu, my_ps, e) * R + rr) * LL;
#pragma unroll
        for (int q = 0; q < NLN; q++) {
          const int ln = lane + 32 * q;
#pragma unroll
          for (int k = 0; k < L; k++) {
            const C m = ln < L * L ? Lp[ln * L + k] : czero<C>();
            in[q][k] = (hf && ln < L * L) ? cmul(sgq[ln * L + k], m) : m;
          }
        }
      }
      C res[NLN][L];
      S::run(sg0, sg1, sg2i, in, sbuf[warp], res, lane);
      if (hf) {
        C ph;
        ph.x = __shfl_sync(0xffffffffu, my_ph.x, e);
        ph.y = __shfl_sync(0xffffffffu, my_ph.y, e);
#pragma unroll
        for (int q = 0; q < NLN; q++) {
          const int ln = lane + 32 * q;
          if (ln < L * L)
#pragma unroll
            for (int k = 0; k < L; k++) cfma(acc[q][k], ph, cmulc(sg[k * L * L + ln], res[q][k]));
        }
      } else {
#pragma unroll
        for (int q = 0; q < NLN; q++)
#pragma unroll
          for (int k = 0; k < L; k++) {
            acc[q][k].x += res[q][k].x;
            acc[q][k].y += res[q][k].y;
          }
      }
      if (++e == npa) {  // the last parent of right-hand side rr
#pragma unroll
        for (int q = 0; q < NLN; q++) {
          const int ln = lane + 32 * q;
#pragma unroll
          for (int k = 0; k < L; k++) {
            if (ln < L * L) {
              const int64_t l = (cs * R + rr) * LL + k * L * L + ln;
              C o = Lc[l];
              o.x += acc[q][k].x;
              o.y += acc[q][k].y;
              Lc[l] = o;
            }
            acc[q][k] = czero<C>();
          }
        }
        e = 0;
        rr++;
      }
    }
  }
}

// ---------------------------------------------------------------- M2F/F2L --
// Pruned odd-size 3-D DFT (size P = 2L-1) of the zero-padded expansion
// (circulant.hpp:96-106: M sits at the low corner of the P^3 grid):
//   F[k0,k1,k2] = sum_{a,b,c<L} M[a,b,c] w^(k0 a + k1 b + k2 c),  w = e^{-2 pi i/P}
// One warp per expansion (several per CTA); each axis pass gives one lane one
// line (its L inputs in registers, its P outputs computed from them).
template <typename T, int L>
struct M2FCfg {
  typedef typename cpx_t<T>::type C;
  static constexpr int P = 2 * L - 1, LL = L * L * L;
  static constexpr int PER_WARP = LL + L * L * P + L * P * P;  // complex elements
  // warps per CTA so that a CTA's shared memory stays within ~48 KB
  static constexpr int NW0 = (int)(49152 / (PER_WARP * sizeof(C)));
  static constexpr int NW = NW0 < 1 ? 1 : (NW0 > 8 ? 8 : NW0);
};

template <typename T, int L>
__global__ void __launch_bounds__(256) k_m2f(int64_t n, const typename cpx_t<T>::type* __restrict__ M,
                                             typename cpx_t<T>::type* __restrict__ F) {
  typedef typename cpx_t<T>::type C;
  constexpr int P = 2 * L - 1, LL = L * L * L, PP = P * P * P;
  constexpr int NW = M2FCfg<T, L>::NW, PER = M2FCfg<T, L>::PER_WARP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* Mi = reinterpret_cast<C*>(smem_raw) + warp * PER;
  C* A = Mi + LL;
  C* B = A + L * L * P;
  // the next expansion is loaded into registers while the current one is
  // transformed
  constexpr int NV = (LL + 31) / 32;
  const int64_t e0 = (int64_t)blockIdx.x * NW + warp, de = (int64_t)gridDim.x * NW;
  C nx[NV];
  if (e0 < n) {
#pragma unroll
    for (int m = 0; m < NV; m++) {
      const int i = lane + 32 * m;
      nx[m] = i < LL ? M[e0 * LL + i] : czero<C>();
    }
  }
  for (int64_t e = e0; e < n; e += de) {
    __syncwarp();
#pragma unroll
    for (int m = 0; m < NV; m++) {
      const int i = lane + 32 * m;
      if (i < LL) Mi[i] = nx[m];
    }
    __syncwarp();
    if (e + de < n) {
#pragma unroll
      for (int m = 0; m < NV; m++) {
        const int i = lane + 32 * m;
        if (i < LL) nx[m] = M[(e + de) * LL + i];
      }
    }
    for (int ln = lane; ln < L * L; ln += 32) {  // axis 2: (a,b) lines
      C v[L];
#pragma unroll
      for (int c = 0; c < L; c++) v[c] = Mi[ln * L + c];
#pragma unroll
      for (int k2 = 0; k2 < P; k2++) {
        C acc = v[0];
#pragma unroll
        for (int c = 1; c < L; c++) cfma(acc, v[c], ctw<T, L>((k2 * c) % P));
        A[ln * P + k2] = acc;
      }
    }
    __syncwarp();
    for (int ln = lane; ln < L * P; ln += 32) {  // axis 1: (a,k2) lines
      const int a = ln / P, k2 = ln % P;
      C v[L];
#pragma unroll
      for (int b = 0; b < L; b++) v[b] = A[(a * L + b) * P + k2];
#pragma unroll
      for (int k1 = 0; k1 < P; k1++) {
        C acc = v[0];
#pragma unroll
        for (int b = 1; b < L; b++) cfma(acc, v[b], ctw<T, L>((k1 * b) % P));
        B[(a * P + k1) * P + k2] = acc;
      }
    }
    __syncwarp();
    for (int ln = lane; ln < P * P; ln += 32) {  // axis 0: (k1,k2) lines
      C v[L];
#pragma unroll
      for (int a = 0; a < L; a++) v[a] = B[a * P * P + ln];
#pragma unroll
      for (int k0 = 0; k0 < P; k0++) {
        C acc = v[0];
#pragma unroll
        for (int a = 1; a < L; a++) cfma(acc, v[a], ctw<T, L>((k0 * a) % P));
        F[e * PP + k0 * P * P + ln] = acc;
      }
    }
  }
}

// Gather the permuted spectra used by M2L once (permutations.hpp:128-150):
// U_k[i] = tables[key_k >> 6][perm[key_k & 63][i]].
template <typename T>
__global__ void k_permute_tables(int64_t n, int PP, const uint32_t* __restrict__ key, const uint16_t* __restrict__ perm,
                                 const typename cpx_t<T>::type* __restrict__ tables,
                                 typename cpx_t<T>::type* __restrict__ out) {
  for (int64_t k = blockIdx.x; k < n; k += gridDim.x) {
    const uint32_t kk = key[k];
    const typename cpx_t<T>::type* U = tables + (int64_t)(kk >> 6) * PP;
    const uint16_t* pm = perm + (int64_t)(kk & 63) * PP;
    for (int i = threadIdx.x; i < PP; i += blockDim.x) out[k * PP + i] = U[pm[i]];
  }
}

// -------------------------------------------------------------- M2L + F2L --
// Inverse DFT of one target slot's spectrum J (acc, K values per thread) into
// its local expansion (fourier2geom, circulant.hpp:109-118):
//   L_t[a,b,c] += (1/PP) sum_k J[k] conj(w)^(k0 a + k1 b + k2 c)
// pruned to a,b,c < L, one line per thread per axis pass in shared memory.
// Safe to call twice in a row: each pass reads only what the previous pass
// wrote after the barrier between them.
template <typename T, int L, int NT>
__device__ __forceinline__ void m2l_f2l(const typename cpx_t<T>::type* acc, typename cpx_t<T>::type* Js,
                                        typename cpx_t<T>::type* Cb, typename cpx_t<T>::type* D,
                                        typename cpx_t<T>::type* __restrict__ Lt) {
  typedef typename cpx_t<T>::type C;
  constexpr int PD = 2 * L - 1, PP = PD * PD * PD, K = (PP + NT - 1) / NT;
  const T inv = T(1) / T(PP);
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int i = threadIdx.x + k * NT;
    if (i < PP) Js[i] = acc[k];
  }
  __syncthreads();
  for (int ln = threadIdx.x; ln < PD * PD; ln += NT) {  // axis 0: (k1,k2) lines -> a
    C v[PD];
#pragma unroll
    for (int k0 = 0; k0 < PD; k0++) v[k0] = Js[k0 * PD * PD + ln];
#pragma unroll
    for (int a = 0; a < L; a++) {
      C s = v[0];
#pragma unroll
      for (int k0 = 1; k0 < PD; k0++) cfmac(s, v[k0], ctw<T, L>((k0 * a) % PD));
      Cb[a * PD * PD + ln] = s;
    }
  }
  __syncthreads();
  for (int ln = threadIdx.x; ln < L * PD; ln += NT) {  // axis 1: (a,k2) lines -> b
    const int a = ln / PD, k2 = ln % PD;
    C v[PD];
#pragma unroll
    for (int k1 = 0; k1 < PD; k1++) v[k1] = Cb[(a * PD + k1) * PD + k2];
#pragma unroll
    for (int b = 0; b < L; b++) {
      C s = v[0];
#pragma unroll
      for (int k1 = 1; k1 < PD; k1++) cfmac(s, v[k1], ctw<T, L>((k1 * b) % PD));
      D[(a * L + b) * PD + k2] = s;
    }
  }
  __syncthreads();
  for (int ln = threadIdx.x; ln < L * L; ln += NT) {  // axis 2: (a,b) lines -> c
    C v[PD];
#pragma unroll
    for (int k2 = 0; k2 < PD; k2++) v[k2] = D[ln * PD + k2];
#pragma unroll
    for (int c = 0; c < L; c++) {
      C s = v[0];
#pragma unroll
      for (int k2 = 1; k2 < PD; k2++) cfmac(s, v[k2], ctw<T, L>((k2 * c) % PD));
      C o = Lt[ln * L + c];
      o.x += s.x * inv;
      o.y += s.y * inv;
      Lt[ln * L + c] = o;
    }
  }
}

// The same for the RB spectra of one target slot at once (acc[k RB + b]: the
// K values of right-hand side b), their local expansions at Lt + b LL: each
// axis pass runs over the lines of all RB spectra, so the CTA's threads stay
// busy and the transform takes three barriers instead of 3 RB.  Every
// output is computed by the operations of m2l_f2l for its spectrum.
template <typename T, int L, int NT, int RB>
__device__ __forceinline__ void m2l_f2l_rhs(const typename cpx_t<T>::type* acc, typename cpx_t<T>::type* Js,
                                            typename cpx_t<T>::type* Cb, typename cpx_t<T>::type* D,
                                            typename cpx_t<T>::type* __restrict__ Lt) {
  typedef typename cpx_t<T>::type C;
  constexpr int PD = 2 * L - 1, PP = PD * PD * PD, K = (PP + NT - 1) / NT, LL = L * L * L;
  constexpr int NB = L * PD * PD, ND = L * L * PD;  // per spectrum: Cb, D elements
  const T inv = T(1) / T(PP);
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int i = threadIdx.x + k * NT;
    if (i < PP)
#pragma unroll
      for (int b = 0; b < RB; b++) Js[b * PP + i] = acc[k * RB + b];
  }
  __syncthreads();
  for (int x = threadIdx.x; x < RB * PD * PD; x += NT) {  // axis 0: (k1,k2) lines -> a
    const int b = x / (PD * PD), ln = x % (PD * PD);
    const C* J = Js + b * PP;
    C* Cq = Cb + b * NB;
    C v[PD];
#pragma unroll
    for (int k0 = 0; k0 < PD; k0++) v[k0] = J[k0 * PD * PD + ln];
#pragma unroll
    for (int a = 0; a < L; a++) {
      C s = v[0];
#pragma unroll
      for (int k0 = 1; k0 < PD; k0++) cfmac(s, v[k0], ctw<T, L>((k0 * a) % PD));
      Cq[a * PD * PD + ln] = s;
    }
  }
  __syncthreads();
  for (int x = threadIdx.x; x < RB * L * PD; x += NT) {  // axis 1: (a,k2) lines -> b
    const int r = x / (L * PD), ln = x % (L * PD);
    const int a = ln / PD, k2 = ln % PD;
    const C* Cq = Cb + r * NB;
    C* Dq = D + r * ND;
    C v[PD];
#pragma unroll
    for (int k1 = 0; k1 < PD; k1++) v[k1] = Cq[(a * PD + k1) * PD + k2];
#pragma unroll
    for (int b = 0; b < L; b++) {
      C s = v[0];
#pragma unroll
      for (int k1 = 1; k1 < PD; k1++) cfmac(s, v[k1], ctw<T, L>((k1 * b) % PD));
      Dq[(a * L + b) * PD + k2] = s;
    }
  }
  __syncthreads();
  for (int x = threadIdx.x; x < RB * L * L; x += NT) {  // axis 2: (a,b) lines -> c
    const int r = x / (L * L), ln = x % (L * L);
    const C* Dq = D + r * ND;
    C* Lq = Lt + r * LL;
    C v[PD];
#pragma unroll
    for (int k2 = 0; k2 < PD; k2++) v[k2] = Dq[ln * PD + k2];
#pragma unroll
    for (int c = 0; c < L; c++) {
      C s = v[0];
#pragma unroll
      for (int k2 = 1; k2 < PD; k2++) cfmac(s, v[k2], ctw<T, L>((k2 * c) % PD));
      C o = Lq[ln * L + c];
      o.x += s.x * inv;
      o.y += s.y * inv;
      Lq[ln * L + c] = o;
    }
  }
}

// One CTA per target slot of a cone batch (M2L.hpp:115-157 target-stationary,
// then the inverse DFT above):
//   J[i] = sum_{(s, k) in list(t)} U_k[i] F_s[i]          (registers)
// J never leaves the SM.
template <typename T, int L, int NT>
__global__ void __launch_bounds__(NT, (sizeof(T) == 8 ? 512 : 1024) / NT) k_m2l(DevPlan P, int64_t t0, int64_t t1, int64_t f0, int64_t f1,
                                                       const typename cpx_t<T>::type* __restrict__ F,
                                                       const typename cpx_t<T>::type* __restrict__ ptab,
                                                       typename cpx_t<T>::type* __restrict__ Lx,
                                                       unsigned long long* __restrict__ queue) {
  typedef typename cpx_t<T>::type C;
  constexpr int PD = 2 * L - 1, LL = L * L * L, PP = PD * PD * PD, K = (PP + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Js = reinterpret_cast<C*>(smem_raw);
  C* Cb = Js + PP;
  C* D = Cb + L * PD * PD;
  __shared__ int64_t cur;
  // target slots are taken in order from a queue, so the slots in flight
  // stay a contiguous window of one cone (good L2 reuse of F and U)
  for (;;) {
    __syncthreads();  // the previous slot's inverse DFT is done with Js/Cb/D
    if (threadIdx.x == 0) cur = t0 + (int64_t)atomicAdd(queue, 1ULL);
    __syncthreads();
    const int64_t t = cur;
    if (t >= t1) break;
    const int64_t eb = P.m2l_ptr[t], ee = P.m2l_ptr[t + 1];
    C acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = czero<C>();
#pragma unroll 2
    for (int64_t e = eb; e < ee; e++) {
      const int64_t src = P.m2l_src[e];
      if (src < f0 || src >= f1) {  // entry outside this cone batch: a plan bug
        if (threadIdx.x == 0) atomicExch(P.err, 1);
        continue;
      }
      const C* Fs = F + (src - f0) * PP;
      const C* U = ptab + (int64_t)P.m2l_tab[e] * PP;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const int i = threadIdx.x + k * NT;
        if (i < PP) cfma(acc[k], __ldg(U + i), __ldg(Fs + i));
      }
    }
    m2l_f2l<T, L, NT>(acc, Js, Cb, D, Lx + t * LL);
  }
}

// Two consecutive target slots per CTA.  Each slot's list is sorted by
// source slot, so a merge of the two lists finds their common sources
// (about a third of the pairs at order 5), whose spectrum F_s is then read
// once for both.  Every accumulator sees its own list in list order with the
// same operations as k_m2l, so the results are bit-identical to it.
template <typename T, int L, int NT>
__global__ void __launch_bounds__(NT, (sizeof(T) == 8 ? 512 : 1024) / NT) k_m2l_pair(DevPlan P, int64_t t0, int64_t t1, int64_t f0, int64_t f1,
                                                            const typename cpx_t<T>::type* __restrict__ F,
                                                            const typename cpx_t<T>::type* __restrict__ ptab,
                                                            typename cpx_t<T>::type* __restrict__ Lx,
                                                            unsigned long long* __restrict__ queue) {
  typedef typename cpx_t<T>::type C;
  constexpr int PD = 2 * L - 1, LL = L * L * L, PP = PD * PD * PD, K = (PP + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Js = reinterpret_cast<C*>(smem_raw);
  C* Cb = Js + PP;
  C* D = Cb + L * PD * PD;
  __shared__ int64_t cur;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) cur = t0 + 2 * (int64_t)atomicAdd(queue, 1ULL);
    __syncthreads();
    const int64_t t = cur;
    if (t >= t1) break;
    const bool two = t + 1 < t1;
    int64_t a = P.m2l_ptr[t], b = P.m2l_ptr[t + 1];
    const int64_t ae = b, be = two ? P.m2l_ptr[t + 2] : b;
    C acc0[K], acc1[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc0[k] = acc1[k] = czero<C>();
    while (a < ae || b < be) {
      const int64_t sa = a < ae ? (int64_t)P.m2l_src[a] : INT64_MAX;
      const int64_t sb = b < be ? (int64_t)P.m2l_src[b] : INT64_MAX;
      const int64_t src = sa < sb ? sa : sb;
      if (src < f0 || src >= f1) {  // entry outside this cone batch: a plan bug
        if (threadIdx.x == 0) atomicExch(P.err, 1);
        if (sa == src) a++;
        if (sb == src) b++;
        continue;
      }
      const C* Fs = F + (src - f0) * PP;
      if (sa == sb) {
        const C* U0 = ptab + (int64_t)P.m2l_tab[a] * PP;
        const C* U1 = ptab + (int64_t)P.m2l_tab[b] * PP;
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int i = threadIdx.x + k * NT;
          if (i < PP) {
            const C f = __ldg(Fs + i);
            cfma(acc0[k], __ldg(U0 + i), f);
            cfma(acc1[k], __ldg(U1 + i), f);
          }
        }
        a++;
        b++;
      } else if (sa < sb) {
        const C* U0 = ptab + (int64_t)P.m2l_tab[a] * PP;
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int i = threadIdx.x + k * NT;
          if (i < PP) cfma(acc0[k], __ldg(U0 + i), __ldg(Fs + i));
        }
        a++;
      } else {
        const C* U1 = ptab + (int64_t)P.m2l_tab[b] * PP;
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int i = threadIdx.x + k * NT;
          if (i < PP) cfma(acc1[k], __ldg(U1 + i), __ldg(Fs + i));
        }
        b++;
      }
    }
    m2l_f2l<T, L, NT>(acc0, Js, Cb, D, Lx + t * LL);
    if (two) m2l_f2l<T, L, NT>(acc1, Js, Cb, D, Lx + (t + 1) * LL);
  }
}

// Right-hand-side blocks: R charge vectors per pass, F and L holding R
// expansions per slot (F + ((s - f0) R + r) PP, Lx + (t R + r) LL).  A CTA
// takes one (target slot, block of RB right-hand sides) at a time; each
// transfer spectrum entry U_k[i] is loaded once and multiplied into the RB
// spectra of its source slot, so the spectra traffic per right-hand side is
// e P^3 (1 + 1/RB) per far pair instead of 2 e P^3.
// CTAs per SM of k_m2l_rhs: room for K x RB complex accumulators per thread
template <typename T, int NT, int RB>
constexpr int m2l_rhs_ctas() {
  return (sizeof(T) == 8 ? (RB >= 8 ? 512 : (RB >= 2 ? 768 : 1024)) : (RB >= 8 ? 768 : 1024)) / NT;
}
// FP32, orders <= 5, up to 4 right-hand sides per CTA: the inverse DFTs of
// a target slot's RB spectra run together (m2l_f2l_rhs, RB workspaces in
// shared memory, 43.5 KB at order 5, so 4 CTAs per SM still fit);
// otherwise one after another
template <typename T, int L, int RB>
__host__ __device__ constexpr bool m2l_rhs_joint() {
  return sizeof(T) == 4 && L <= 5 && RB > 1 && RB <= 4;
}

template <typename T, int L, int NT, int RB>
__global__ void __launch_bounds__(NT, m2l_rhs_ctas<T, NT, RB>()) k_m2l_rhs(DevPlan P, int64_t t0, int64_t t1, int64_t f0, int64_t f1, int R,
                                                             const typename cpx_t<T>::type* __restrict__ F,
                                                             const typename cpx_t<T>::type* __restrict__ ptab,
                                                             typename cpx_t<T>::type* __restrict__ Lx,
                                                             unsigned long long* __restrict__ queue) {
  typedef typename cpx_t<T>::type C;
  constexpr int PD = 2 * L - 1, LL = L * L * L, PP = PD * PD * PD, K = (PP + NT - 1) / NT;
  constexpr bool JOINT = m2l_rhs_joint<T, L, RB>();
  constexpr int MS = JOINT ? RB : 1;  // inverse-DFT workspaces
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Js = reinterpret_cast<C*>(smem_raw);
  C* Cb = Js + MS * PP;
  C* D = Cb + MS * L * PD * PD;
  __shared__ int64_t cur;
  const int nb = R / RB;
  const int64_t nwork = (t1 - t0) * nb;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) cur = (int64_t)atomicAdd(queue, 1ULL);
    __syncthreads();
    const int64_t w = cur;
    if (w >= nwork) break;
    const int64_t t = t0 + w / nb;
    const int r0 = (int)(w % nb) * RB;
    const int64_t eb = P.m2l_ptr[t], ee = P.m2l_ptr[t + 1];
    C acc[K][RB];
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int b = 0; b < RB; b++) acc[k][b] = czero<C>();
    for (int64_t e = eb; e < ee; e++) {
      const int64_t src = P.m2l_src[e];
      if (src < f0 || src >= f1) {  // entry outside this cone batch: a plan bug
        if (threadIdx.x == 0) atomicExch(P.err, 1);
        continue;
      }
      const C* Fs = F + ((src - f0) * R + r0) * PP;
      const C* U = ptab + (int64_t)P.m2l_tab[e] * PP;
#pragma unroll
      for (int k = 0; k < K; k++) {
        const int i = threadIdx.x + k * NT;
        if (i < PP) {
          const C u = __ldg(U + i);
#pragma unroll
          for (int b = 0; b < RB; b++) cfma(acc[k][b], u, __ldg(Fs + b * PP + i));
        }
      }
    }
    if constexpr (JOINT) {
      m2l_f2l_rhs<T, L, NT, RB>(&acc[0][0], Js, Cb, D, Lx + (t * R + r0) * LL);
    } else {
#pragma unroll
      for (int b = 0; b < RB; b++) {
        C a[K];
#pragma unroll
        for (int k = 0; k < K; k++) a[k] = acc[k][b];
        m2l_f2l<T, L, NT>(a, Js, Cb, D, Lx + (t * R + r0 + b) * LL);
      }
    }
  }
}

// Right-hand-side blocks with target groups, fed through shared memory by
// bulk copies (FP32 spectra).  A work item is (G consecutive target slots of
// a cone batch, RB right-hand sides).  Their lists are sorted by source slot;
// merged, every source slot met by any of the G lists is one entry, and its
// RB spectra F_s are loaded once for all the targets that meet it (a group of
// 4 consecutive slots meets 0.45 distinct sources per far pair on a sphere
// at 40 points per wavelength squared, order 5), with the transfer spectrum
// U_k of each such pair.
//
// Warp roles: the last warp produces, the others consume.  The producer
// takes work items from the queue, loads the G lists into shared memory,
// merges them and, per entry, copies the RB spectra of the source and the
// entry's transfer spectra into one of NS stages with 1-D bulk copies
// (cp.async.bulk global -> shared, completing on the stage's "full"
// mbarrier).  Consumer thread c owns spectrum entries c + k NC and keeps the
// G x RB accumulators of its entries in registers; after a stage it arrives
// on the stage's "empty" mbarrier, and after the last entry of an item it
// runs the inverse DFT of every (target, right-hand side) with an entry,
// NSPEC spectra per round, and adds the results into L.  The producer keeps
// filling stages meanwhile.
//
// Every accumulator sees its list in list order with the operations of
// k_m2l_rhs, and the inverse DFT sums in the order of m2l_f2l, so the
// results are bit-identical to k_m2l_rhs (and to the one-right-hand-side
// kernels).  A copy starts at the 16-byte boundary at or below its first
// byte and ends at the one at or above its last (both buffers carry 16 bytes
// of slack at the end); consumers index from the remainder.
//
// Every wait is bounded.  A thread that gives up sets a shared stop flag
// (the other waits then return at once) and the error code 3; the producer
// then waits (bounded) for the copies it issued before it returns.
template <int L>
struct M2LBulk {
  static constexpr int PD = 2 * L - 1, PP = PD * PD * PD, LL = L * L * L;
  static constexpr int G = kM2LGroup;                                   // target slots per work item
  static constexpr int RB = L <= 5 ? 4 : 2;                             // right-hand sides per work item
  static constexpr int K = (PP + 767) / 768;                            // entries per consumer thread
  static constexpr int NC = 32 * ((PP + 32 * K - 1) / (32 * K));        // consumer threads
  static constexpr int NT = NC + 32;                                    // + the producer warp
  static constexpr int NSPEC = L <= 5 ? 4 : 1;                          // spectra per inverse-DFT round
  static constexpr int FB = (RB * PP * 8 + 16 + 15) / 16 * 16;          // stage bytes of the F block
  static constexpr int UB = (PP * 8 + 16 + 15) / 16 * 16;               // stage bytes of one U
  static constexpr int SB = FB + G * UB;
  static constexpr int XB = NSPEC * (PP + L * PD * PD + L * L * PD) * 8;  // inverse-DFT scratch
  static constexpr int LCAP = L <= 4 ? 1024 : 2048;                     // list entries of one work item
  static constexpr int HDR = 1024;                                      // barriers, entry records, twiddles
  static constexpr int NS0 = (232448 - XB - LCAP * 8 - HDR) / SB;
  static constexpr int NS = NS0 > 4 ? 4 : NS0;                          // stages
  static constexpr int CTAS = L <= 3 ? 4 : (L == 4 ? 2 : 1);           // CTAs per SM
  static constexpr size_t smem() { return (size_t)NS * SB + XB + (size_t)LCAP * 8 + HDR; }
};

struct BulkEntry {  // one stage's record, written by the producer
  int64_t tb;       // first target slot of the item
  int mask;         // targets of the item that meet this source
  int flags;        // 1: last entry of the item; 2: no more work
  int nt, r0;       // targets in the item, first right-hand side
  int foff;         // F block: offset (complex entries) from the stage start
  int uoff[kM2LGroup];
};

constexpr uint32_t kBulkWait = 1u << 22;  // polls before a wait counts as failed

template <int L>
__global__ void __launch_bounds__(M2LBulk<L>::NT, M2LBulk<L>::CTAS) k_m2l_bulk(
    DevPlan P, int64_t t0, int64_t t1, int64_t f0, int64_t f1, int R, const float2* __restrict__ F,
    const float2* __restrict__ ptab, float2* __restrict__ Lx, unsigned long long* __restrict__ queue) {
  typedef M2LBulk<L> B;
  constexpr int PD = B::PD, PP = B::PP, LL = B::LL, G = B::G, RB = B::RB, K = B::K, NC = B::NC, NS = B::NS,
                NSPEC = B::NSPEC, FB = B::FB, UB = B::UB, SB = B::SB;
  static_assert(NS >= 2, "at least two stages");
  static_assert((G * RB) % NSPEC == 0, "whole inverse-DFT rounds");
  static_assert(NSPEC * LL <= NC, "one output of the last inverse-DFT pass per thread");
  static_assert(NS * 16 + 8 + NS * sizeof(BulkEntry) + PD * 8 + 8 <= B::HDR, "header");
  extern __shared__ __align__(16) unsigned char smem_raw[];  // stage offsets are multiples of 16 bytes
  unsigned char* stages = smem_raw;
  float2* Js = reinterpret_cast<float2*>(smem_raw + NS * SB);
  float2* Cb = Js + NSPEC * PP;
  float2* D = Cb + NSPEC * L * PD * PD;
  int32_t* ls_src = reinterpret_cast<int32_t*>(D + NSPEC * L * L * PD);
  uint32_t* ls_tab = reinterpret_cast<uint32_t*>(ls_src + B::LCAP);
  uint64_t* full = reinterpret_cast<uint64_t*>(ls_tab + B::LCAP);
  uint64_t* empty = full + NS;
  uint64_t* cbar = empty + NS;
  BulkEntry* rec = reinterpret_cast<BulkEntry*>(cbar + 1);
  float2* tw = reinterpret_cast<float2*>(rec + NS);
  volatile int* stop = reinterpret_cast<volatile int*>(tw + PD);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr unsigned kAll = 0xffffffffu;
  if (tid == 0) {
    for (int i = 0; i < NS; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], NC / 32);
    }
    mbar_init(cbar, NC / 32);
    *stop = 0;
  }
  if (tid < PD) tw[tid] = ctw<float, L>(tid);
  __syncthreads();

  if (warp == NC / 32) {
    // ---------------------------------------------------------- producer
    const int nb = R / RB;
    const int64_t nwork = (t1 - t0 + G - 1) / G * nb;
    uint32_t it = 0;  // stages issued
    bool ok = true;
    for (;;) {
      unsigned long long w = 0;
      if (lane == 0) w = atomicAdd(queue, 1ULL);
      w = __shfl_sync(kAll, w, 0);
      if ((int64_t)w >= nwork) break;
      const int64_t tb = t0 + (int64_t)(w / nb) * G;
      const int r0 = (int)(w % nb) * RB;
      const int nt = (int)(t1 - tb < G ? t1 - tb : G);
      const int64_t eb = P.m2l_ptr[tb], ee = P.m2l_ptr[tb + nt];
      const int64_t n = ee - eb;
      if (n == 0) continue;
      if (n > B::LCAP) {  // the launcher checks the plan's largest group: a plan bug
        if (lane == 0) atomicExch(P.err, 1);
        continue;
      }
      __syncwarp();  // lane 0 is done with the previous item's lists
      for (int64_t i = lane; i < n; i += 32) {
        ls_src[i] = P.m2l_src[eb + i];
        ls_tab[i] = P.m2l_tab[eb + i];
      }
      __syncwarp();
      if (lane == 0) {
        int hd[G], he[G];
#pragma unroll
        for (int j = 0; j < G; j++) {
          hd[j] = j < nt ? (int)(P.m2l_ptr[tb + j] - eb) : 0;
          he[j] = j < nt ? (int)(P.m2l_ptr[tb + j + 1] - eb) : 0;
        }
        // one entry of look-ahead, so the item's last entry is known when issued
        bool have = false;
        int pmask = 0, psrc = 0;
        uint32_t ptabs[G];
        auto issue = [&](bool last) -> bool {
          const int s = (int)(it % NS);
          const uint32_t ph = (it / NS) & 1u;
          if (!mbar_wait_or_stop(&empty[s], ph ^ 1u, kBulkWait, stop)) return false;
          unsigned char* st = stages + (size_t)s * SB;
          BulkEntry& e = rec[s];
          const uintptr_t a = (uintptr_t)(F + ((int64_t)(psrc - f0) * R + r0) * PP);
          const uintptr_t a0 = a & ~(uintptr_t)15, a1 = (a + (uintptr_t)RB * PP * 8 + 15) & ~(uintptr_t)15;
          uint32_t total = (uint32_t)(a1 - a0);
          e.tb = tb;
          e.mask = pmask;
          e.flags = last ? 1 : 0;
          e.nt = nt;
          e.r0 = r0;
          e.foff = (int)((a - a0) >> 3);
          uintptr_t u0[G];
          uint32_t ub[G];
#pragma unroll
          for (int j = 0; j < G; j++) {
            u0[j] = 0;
            ub[j] = 0;
            if ((pmask >> j) & 1) {
              const uintptr_t u = (uintptr_t)(ptab + (int64_t)ptabs[j] * PP);
              u0[j] = u & ~(uintptr_t)15;
              ub[j] = (uint32_t)(((u + (uintptr_t)PP * 8 + 15) & ~(uintptr_t)15) - u0[j]);
              e.uoff[j] = (int)((u - u0[j]) >> 3);
              total += ub[j];
            }
          }
          mbar_arrive_expect_tx(&full[s], total);
          bulk_g2s(st, (const void*)a0, (uint32_t)(a1 - a0), &full[s]);
#pragma unroll
          for (int j = 0; j < G; j++)
            if ((pmask >> j) & 1) bulk_g2s(st + FB + j * UB, (const void*)u0[j], ub[j], &full[s]);
          it++;
          return true;
        };
        for (;;) {
          int src = INT_MAX;
#pragma unroll
          for (int j = 0; j < G; j++)
            if (hd[j] < he[j] && ls_src[hd[j]] < src) src = ls_src[hd[j]];
          if (src == INT_MAX) break;
          int mask = 0;
          uint32_t tabs[G];
#pragma unroll
          for (int j = 0; j < G; j++) {
            tabs[j] = 0;
            if (hd[j] < he[j] && ls_src[hd[j]] == src) {
              mask |= 1 << j;
              tabs[j] = ls_tab[hd[j]];
              hd[j]++;
            }
          }
          if (src < f0 || src >= f1) {  // entry outside this cone batch: a plan bug
            atomicExch(P.err, 1);
            continue;
          }
          if (have && !issue(false)) {
            ok = false;
            break;
          }
          have = true;
          psrc = src;
          pmask = mask;
#pragma unroll
          for (int j = 0; j < G; j++) ptabs[j] = tabs[j];
        }
        if (ok && have && !issue(true)) ok = false;
      }
      ok = __shfl_sync(kAll, ok, 0);
      if (!ok) break;
    }
    if (lane == 0) {
      if (ok) {  // no more work
        const int s = (int)(it % NS);
        if (mbar_wait_or_stop(&empty[s], ((it / NS) & 1u) ^ 1u, kBulkWait, stop)) {
          rec[s].flags = 2;
          mbar_arrive(&full[s]);
        } else {
          ok = false;
        }
      }
      if (!ok) {
        *stop = 1;
        atomicExch(P.err, 3);
        // the copies issued into the last NS stages land before the CTA ends
        for (uint32_t k = it > (uint32_t)NS ? it - NS : 0; k < it; k++) mbar_wait(&full[k % NS], (k / NS) & 1u, kBulkWait);
      }
    }
    return;
  }

  // ------------------------------------------------------------ consumers
  float2 acc[G][RB][K];
#pragma unroll
  for (int j = 0; j < G; j++)
#pragma unroll
    for (int r = 0; r < RB; r++)
#pragma unroll
      for (int k = 0; k < K; k++) acc[j][r][k] = czero<float2>();
  int seen = 0;
  uint32_t cph = 0;
  const float inv = 1.0f / (float)PP;
  // barrier of the consumer warps (bounded; false once any thread gave up)
  auto cbarrier = [&]() -> bool {
    __syncwarp();
    if (lane == 0) mbar_arrive(cbar);
    const bool ok = __all_sync(kAll, mbar_wait_or_stop(cbar, cph, kBulkWait, stop));
    cph ^= 1u;
    if (!ok && lane == 0) {
      *stop = 1;
      atomicExch(P.err, 3);
    }
    return ok;
  };
  for (uint32_t it = 0;; it++) {
    const int s = (int)(it % NS);
    if (!__all_sync(kAll, mbar_wait_or_stop(&full[s], (it / NS) & 1u, kBulkWait, stop))) {
      if (lane == 0) {
        *stop = 1;
        atomicExch(P.err, 3);
      }
      break;
    }
    const BulkEntry e = rec[s];
    if (e.flags & 2) break;
    const float2* st = reinterpret_cast<const float2*>(stages + (size_t)s * SB);
    const float2* Fs = st + e.foff;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int i = tid + k * NC;
      if (i < PP) {
        float2 f[RB];
#pragma unroll
        for (int r = 0; r < RB; r++) f[r] = Fs[r * PP + i];
#pragma unroll
        for (int j = 0; j < G; j++)
          if ((e.mask >> j) & 1) {
            const float2 u = st[(FB + j * UB) / 8 + e.uoff[j] + i];
#pragma unroll
            for (int r = 0; r < RB; r++) cfma(acc[j][r][k], u, f[r]);
          }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    seen |= e.mask;
    if (!(e.flags & 1)) continue;
    // inverse DFT of every (target, right-hand side) with an entry, the
    // passes of m2l_f2l over NSPEC spectra at a time
    bool ok = true;
#pragma unroll
    for (int q0 = 0; q0 < G * RB; q0 += NSPEC) {
      bool live = false;
#pragma unroll
      for (int sp = 0; sp < NSPEC; sp++) {
        const int j = (q0 + sp) / RB;
        live |= j < e.nt && ((seen >> j) & 1);
      }
      if (!live || !ok) continue;
      // this thread's output of the last pass (one per thread): its L entry
      // is loaded now, so the load overlaps the first two passes
      float2* l3 = nullptr;
      float2 lold = czero<float2>();
      if (tid < NSPEC * LL) {
        const int sp = tid / LL, rem = tid - sp * LL;
        const int q = q0 + sp, j = q / RB, r = q - j * RB;
        if (j < e.nt && ((seen >> j) & 1)) {
          l3 = Lx + ((e.tb + j) * R + e.r0 + r) * LL + rem;
          lold = *l3;
        }
      }
#pragma unroll
      for (int sp = 0; sp < NSPEC; sp++)
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int i = tid + k * NC;
          if (i < PP) Js[sp * PP + i] = acc[(q0 + sp) / RB][(q0 + sp) % RB][k];
        }
      if (!(ok = cbarrier())) continue;
      for (int o = tid; o < NSPEC * L * PD * PD; o += NC) {  // axis 0: (k1,k2) lines -> a
        const int sp = o / (L * PD * PD), rem = o - sp * (L * PD * PD);
        const int a = rem / (PD * PD), ln = rem - a * (PD * PD);
        const float2* v = Js + sp * PP + ln;
        float2 sum = v[0];
#pragma unroll
        for (int k0 = 1; k0 < PD; k0++) cfmac(sum, v[k0 * PD * PD], tw[(k0 * a) % PD]);
        Cb[sp * L * PD * PD + a * PD * PD + ln] = sum;
      }
      if (!(ok = cbarrier())) continue;
      for (int o = tid; o < NSPEC * L * L * PD; o += NC) {  // axis 1: (a,k2) lines -> b
        const int sp = o / (L * L * PD), rem = o - sp * (L * L * PD);
        const int a = rem / (L * PD), rem2 = rem - a * (L * PD);
        const int b = rem2 / PD, k2 = rem2 - b * PD;
        const float2* v = Cb + sp * L * PD * PD + a * PD * PD + k2;
        float2 sum = v[0];
#pragma unroll
        for (int k1 = 1; k1 < PD; k1++) cfmac(sum, v[k1 * PD], tw[(k1 * b) % PD]);
        D[sp * L * L * PD + (a * L + b) * PD + k2] = sum;
      }
      if (!(ok = cbarrier())) continue;
      if (l3) {  // axis 2: (a,b) lines -> c, added into L
        const int sp = tid / LL, rem = tid - sp * LL;
        const int ln = rem / L, c = rem - ln * L;
        const float2* v = D + sp * L * L * PD + ln * PD;
        float2 sum = v[0];
#pragma unroll
        for (int k2 = 1; k2 < PD; k2++) cfmac(sum, v[k2], tw[(k2 * c) % PD]);
        lold.x += sum.x * inv;
        lold.y += sum.y * inv;
        *l3 = lold;
      }
    }
    if (!ok) break;
#pragma unroll
    for (int j = 0; j < G; j++)
#pragma unroll
      for (int r = 0; r < RB; r++)
#pragma unroll
        for (int k = 0; k < K; k++) acc[j][r][k] = czero<float2>();
    seen = 0;
  }
}

// -------------------------------------------------------------------- L2P --
// One CTA (4 warps) per target leaf at a precomputed level
// (dwnpass.hpp:39-47): HF (phfL2P, L2P.hpp:122-142)
//   p_j = sum_d exp(i k d.(x_j - c)) sum_l Z(j, l) sig2_d[l] L_d[l]
// LF (plfL2P :165-173): p_j = sum_l Z(j, l) L[l].  Writes p_far.
// Warps take the leaf's slots in turn, lanes its particles; each lane keeps
// its particle's 3 L basis values in registers and accumulates over the
// warp's slots in registers; the 4 warps are summed at the end.
// Lx: base of the local expansions read here (slot s, right-hand side r at
// Lx + (s R + r) LL); only the leaf slots with a direction in [d0, d1)
// contribute; pfar holds R potentials per particle (pfar[j R + r]), written
// (acc = false) or added to (acc = true).  RC right-hand sides per pass over
// the slots (the phase of a slot is computed once per pass).
template <typename T, int L, int RC>
__global__ void __launch_bounds__(128) k_l2p(DevPlan P, const int32_t* __restrict__ leaves, int nleaves,
                                             const typename cpx_t<T>::type* __restrict__ sig2,
                                             const typename cpx_t<T>::type* __restrict__ Lx,
                                             double2* __restrict__ pfar, int R, int d0, int d1, bool accum) {
  typedef typename cpx_t<T>::type C;
  constexpr int LL = L * L * L;
  __shared__ C buf[4][LL];
  __shared__ double2 part[4][RC][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int li = blockIdx.x; li < nleaves; li += gridDim.x) {
    const int c = leaves[li];
    int64_t sb, se;
    dir_range(P.T_cptr, P.T_cdir, c, d0, d1, &sb, &se);
    if (sb == se) continue;
    const int n = P.T_nprt[c], f = P.T_first[c];
    const double4 ct = P.T_ctr[c];
    const int lv = P.T_lvl[c];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const double* dirs = P.dirs + P.dir_off[h] * 3;
    const C* s2 = sig2 + P.sig_off[h];
    for (int p0 = 0; p0 < n; p0 += 32) {
      const int np = min(32, n - p0);
      const int pi = f + p0 + min(lane, np - 1);
      double xr[3];
      T B[3][L];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        xr[k] = P.T_pos[3 * (int64_t)pi + k] - (&ct.x)[k];
        lagrange_all<L, T>((T)xr[k], (T)ct.w, B[k]);
      }
      for (int r0 = 0; r0 < R; r0 += RC) {
        const int nr = min(RC, R - r0);
        double2 acc[RC];
#pragma unroll
        for (int u = 0; u < RC; u++) acc[u] = make_double2(0., 0.);
        // units (slot of this warp, right-hand side); the next unit's
        // expansion (and, on a new slot, signature) is loaded into registers
        // while the current one is contracted
        constexpr int NV = (LL + 31) / 32;
        const int64_t nunit = ((se - sb - warp + 3) / 4) * nr;
        C nl[NV], ns[NV];
        int nd = 0;
        auto fetch = [&](int64_t k) {
          const int64_t j = sb + warp + 4 * (k / nr);
          const int u = (int)(k % nr);
          const int slot = P.T_cslot[j];
          const C* Ls = Lx + ((int64_t)slot * R + r0 + u) * LL;
#pragma unroll
          for (int m = 0; m < NV; m++) {
            const int l = lane + 32 * m;
            nl[m] = l < LL ? Ls[l] : czero<C>();
          }
          if (u == 0) {
            nd = P.T_cdir[j];
            const C* Ss = s2 + (int64_t)(hf ? nd : 0) * LL;
#pragma unroll
            for (int m = 0; m < NV; m++) {
              const int l = lane + 32 * m;
              ns[m] = (hf && l < LL) ? Ss[l] : czero<C>();
            }
          }
        };
        if (nunit > 0) fetch(0);
        C ph = czero<C>();
        for (int64_t k = 0; k < nunit; k++) {
          const int u = (int)(k % nr);
          if (u == 0 && hf) {
            const double* dv = dirs + 3 * nd;
            ph = expi<C>(P.kappa * (dv[0] * xr[0] + dv[1] * xr[1] + dv[2] * xr[2]));
          }
          __syncwarp();
#pragma unroll
          for (int m = 0; m < NV; m++) {
            const int l = lane + 32 * m;
            if (l < LL) buf[warp][l] = hf ? cmul(ns[m], nl[m]) : nl[m];
          }
          __syncwarp();
          if (k + 1 < nunit) fetch(k + 1);
          // sum_{a,b,c} B0[a] B1[b] B2[c] X[a,b,c] = sum_a B0[a] (sum_b B1[b] (sum_c B2[c] X[a,b,c]))
          C sum = czero<C>();
#pragma unroll
          for (int a = 0; a < L; a++) {
            C sa = czero<C>();
#pragma unroll
            for (int b = 0; b < L; b++) {
              C sbb = czero<C>();
#pragma unroll
              for (int cc = 0; cc < L; cc++) rfma(sbb, B[2][cc], buf[warp][(a * L + b) * L + cc]);
              rfma(sa, B[1][b], sbb);
            }
            rfma(sum, B[0][a], sa);
          }
          if (hf) sum = cmul(sum, ph);
#pragma unroll
          for (int v = 0; v < RC; v++)
            if (v == u) {
              acc[v].x += (double)sum.x;
              acc[v].y += (double)sum.y;
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < RC; u++) part[warp][u][lane] = acc[u];
        __syncthreads();
        if (threadIdx.x < np) {
#pragma unroll
          for (int u = 0; u < RC; u++) {
            if (r0 + u >= R) break;
            double2 t = part[0][u][threadIdx.x];
            for (int w = 1; w < 4; w++) {
              t.x += part[w][u][threadIdx.x].x;
              t.y += part[w][u][threadIdx.x].y;
            }
            double2* o = pfar + (int64_t)(f + p0 + threadIdx.x) * R + r0 + u;
            if (accum) {
              t.x += o->x;
              t.y += o->y;
            }
            *o = t;
          }
        }
      }
    }
  }
}

// -------------------------------------------------------------------- P2P --
// Mixed-precision near field.  The phase k r needs ~1e-7 rad absolute
// accuracy at k r up to ~1e2, beyond FP32: the difference vector, r^2, r and
// the reduction of k r to [-pi/2, pi/2] (n = rint(k r / pi)) run in FP64;
// sin/cos of the reduced angle are evaluated in FP32 by their Taylor series
// to degree 13/12, 1/(4 pi r) and the complex products in FP32; every
// product is accumulated in FP64.
__device__ __forceinline__ void sincos_reduced(double theta, float& s, float& c) {
  // theta = n pi + x, |x| <= pi/2 (FP64 reduction; n pi exact inside the FMA)
  const double n = rint(theta * 0.31830988618379067154);  // 1/pi
  const float x = (float)fma(-n, 3.14159265358979323846, theta);
  const float x2 = x * x;
  // sin x = x (1 - x^2/3! + ... + x^12/13!), cos x = 1 - x^2/2! + ... + x^12/12!
  // (Taylor; truncation < 7e-10 on [-pi/2, pi/2])
  float ps = fmaf(x2, 1.6059043836821613e-10f, -2.5052108385441720e-08f);
  ps = fmaf(x2, ps, 2.7557319223985893e-06f);
  ps = fmaf(x2, ps, -1.9841269841269841e-04f);
  ps = fmaf(x2, ps, 8.3333333333333333e-03f);
  ps = fmaf(x2, ps, -1.6666666666666667e-01f);
  ps = fmaf(x2, ps, 1.0f);
  float pc = fmaf(x2, 2.0876756987868099e-09f, -2.7557319223985891e-07f);
  pc = fmaf(x2, pc, 2.4801587301587302e-05f);
  pc = fmaf(x2, pc, -1.3888888888888889e-03f);
  pc = fmaf(x2, pc, 4.1666666666666667e-02f);
  pc = fmaf(x2, pc, -0.5f);
  pc = fmaf(x2, pc, 1.0f);
  // (-1)^n on both
  const float sg = (__double2int_rn(n) & 1) ? -1.0f : 1.0f;
  s = sg * x * ps;
  c = sg * pc;
}


// Near field, tiled: one CTA (4 warps) per work item (part of the sources of
// one chunk of <= 32 target particles of one leaf); CTAs take items from a
// global queue in the host's order of decreasing work.  The chunk's source ranges are streamed through shared
// memory in tiles of TS particles loaded with coalesced reads; inside a warp,
// lanes form groups of tp >= nt lanes (one target each) and the 4 warps x
// groups take interleaved sources of the tile, two at a time.  Partial sums
// are reduced in FP64 through shuffles and shared memory; each target is
// written once.
//   MIXED = false: FP64 throughout (P2P.hpp:43-79 arithmetic, p2p_pair64).
//   MIXED = true : difference vector, r^2, 1/r and the reduction of k r in
//   FP64; sin/cos of the reduced angle, 1/(4 pi r) and the complex products
//   in FP32 with compensated sums (p2p_pair_mixed).
// Source record in shared memory: a = (x, y), b = (z, charge) with the FP32
// charge bits in b.y (mixed) or the FP64 charge in c (FP64 path).

// Approximate FP64 reciprocal square root (the PTX instruction
// rsqrt.approx.ftz.f64, about FP32 accuracy); callers refine it by Newton
// steps y <- y (3/2 - R y^2 / 2), each of which doubles the correct bits.
__device__ __forceinline__ double rsqrt_approx64(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

// One FP64 source/target interaction.
__device__ __forceinline__ void p2p_pair64(double x0, double x1, double x2, double2 a, double2 b, double2 qd,
                                           double kappa, double& pr, double& pim) {
  const double pi4m1 = 1. / (4. * 3.14159265358979323846);
  const double dx = x0 - a.x, dy = x1 - a.y, dz = x2 - b.x;
  const double R = fma(dx, dx, fma(dy, dy, dz * dz));
  if (R < 1.e-16) return;  // self / duplicate pairs (P2P.hpp:66)
  // 1/sqrt(R): approximate FP64 estimate, two Newton steps (quadratic)
  double y = rsqrt_approx64(R);
  const double hR = 0.5 * R;
  y = y * fma(-hR * y, y, 1.5);
  y = y * fma(-hR * y, y, 1.5);
  const double rr = y * R * kappa;
  const double K = y * pi4m1;
  double sn_, cs_;
  sincos_cw(rr, sn_, cs_);
  cs_ *= K;
  sn_ *= K;
  pr = fma(cs_, qd.x, fma(-sn_, qd.y, pr));
  pim = fma(cs_, qd.y, fma(sn_, qd.x, pim));
}

// Compensated (Kahan) FP32 summation: s - c carries the sum.
__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
  const float y = x - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// Mixed-precision interaction with FP32 compensated accumulators (the FP64
// path keeps p2p_pair<false>).  1/r: approximate FP64 reciprocal square root
// refined once in FP64 (relative error ~1e-14), used for k r, and rounded to
// FP32 for 1/(4 pi r).  k r = n pi + x with n read from the
// low mantissa bits of k r / pi + 1.5 * 2^52 (exact for k r / pi < 2^51) and
// x = k r - n pi in FP64; sin/cos of x by the FP32 Taylor polynomials of
// sincos_reduced, (-1)^n applied to both.
__device__ __forceinline__ void p2p_pair_mixed(double x0, double x1, double x2, double2 a, double2 b, double kappa,
                                               float& sr, float& cr, float& si, float& ci) {
  const double dx = x0 - a.x, dy = x1 - a.y, dz = x2 - b.x;
  const double R = fma(dx, dx, fma(dy, dy, dz * dz));
  if (R < 1.e-16) return;  // self / duplicate pairs (P2P.hpp:66)
  double yd = rsqrt_approx64(R);
  yd = yd * fma(-0.5 * R * yd, yd, 1.5);
  const float y = (float)yd;
  const double theta = R * yd * kappa;
  const double t = fma(theta, 0.31830988618379067154, 6755399441055744.0);  // + 1.5 * 2^52
  const double n = t - 6755399441055744.0;
  const int odd = __double2loint(t) & 1;
  const float x = (float)fma(-n, 3.14159265358979323846, theta);
  const float xx = x * x;
  float ps = fmaf(xx, 1.6059043836821613e-10f, -2.5052108385441720e-08f);
  ps = fmaf(xx, ps, 2.7557319223985893e-06f);
  ps = fmaf(xx, ps, -1.9841269841269841e-04f);
  ps = fmaf(xx, ps, 8.3333333333333333e-03f);
  ps = fmaf(xx, ps, -1.6666666666666667e-01f);
  ps = fmaf(xx, ps, 1.0f);
  float pc = fmaf(xx, 2.0876756987868099e-09f, -2.7557319223985891e-07f);
  pc = fmaf(xx, pc, 2.4801587301587302e-05f);
  pc = fmaf(xx, pc, -1.3888888888888889e-03f);
  pc = fmaf(xx, pc, 4.1666666666666667e-02f);
  pc = fmaf(xx, pc, -0.5f);
  pc = fmaf(xx, pc, 1.0f);
  const float K = odd ? -0.0795774715459476679f * y : 0.0795774715459476679f * y;  // (-1)^n / (4 pi r)
  const float c = pc * K, s = x * ps * K;
  const float2 q = *reinterpret_cast<const float2*>(&b.y);
  kahan_add(sr, cr, fmaf(c, q.x, -s * q.y));
  kahan_add(si, ci, fmaf(c, q.y, s * q.x));
}

template <bool MIXED>
__global__ void __launch_bounds__(128) k_p2p_tiled(DevPlan P, int64_t nitem, const int32_t* __restrict__ order,
                                                   const int32_t* __restrict__ item_chunk,
                                                   const int32_t* __restrict__ tfirst, const int32_t* __restrict__ tn,
                                                   const int64_t* __restrict__ ptr, const int32_t* __restrict__ sfirst,
                                                   const int32_t* __restrict__ sn, const void* __restrict__ qv,
                                                   double2* __restrict__ pnear, double2* __restrict__ tpart,
                                                   unsigned long long* __restrict__ queue) {
  constexpr int TS = 512;
  typedef typename std::conditional<MIXED, float2, double2>::type Q;
  const Q* q = static_cast<const Q*>(qv);
  __shared__ double2 sa[TS], sb[TS];
  __shared__ double2 sc[MIXED ? 1 : TS];
  __shared__ double2 red[4][32];
  __shared__ int64_t cur;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) cur = (int64_t)atomicAdd(queue, 1ULL);
    __syncthreads();
    const int64_t k = cur;
    if (k >= nitem) break;
    const int64_t it = order[k];
    const int64_t ch = item_chunk ? item_chunk[it] : it;
    const int f = tfirst[ch], nt = tn[ch];
    int tp = 1;
    while (tp < nt) tp <<= 1;
    const int groups = 32 / tp, G = 4 * groups;
    const int mt = lane & (tp - 1), gid = warp * groups + lane / tp;
    const int ti = f + min(mt, nt - 1);
    const double x0 = P.T_pos[3 * (int64_t)ti], x1 = P.T_pos[3 * (int64_t)ti + 1], x2 = P.T_pos[3 * (int64_t)ti + 2];
    double pr = 0., pim = 0.;
    float sr = 0.f, cr = 0.f, si = 0.f, ci = 0.f;  // mixed: compensated FP32 sums
    const int64_t rb = ptr[it], re = ptr[it + 1];
    int64_t r = rb;
    int off = 0;  // position inside range r
    while (r < re) {
      // fill one tile from consecutive ranges (uniform control flow)
      int fill = 0;
      __syncthreads();
      while (r < re && fill < TS) {
        const int s0 = sfirst[r], ns = sn[r];
        const int take = min(ns - off, TS - fill);
        for (int t = threadIdx.x; t < take; t += blockDim.x) {
          const int64_t sj = (int64_t)s0 + off + t;
          const double* y = P.S_pos + 3 * sj;
          sa[fill + t] = make_double2(y[0], y[1]);
          if (MIXED) {
            const float2 qq = *reinterpret_cast<const float2*>(&q[sj]);
            double qbits;
            *reinterpret_cast<float2*>(&qbits) = qq;
            sb[fill + t] = make_double2(y[2], qbits);
          } else {
            sb[fill + t] = make_double2(y[2], 0.);
            sc[fill + t] = *reinterpret_cast<const double2*>(&q[sj]);
          }
        }
        fill += take;
        off += take;
        if (off == ns) {
          r++;
          off = 0;
        }
      }
      __syncthreads();
      int j = gid;
      if constexpr (MIXED) {
        for (; j + G < fill; j += 2 * G) {
          p2p_pair_mixed(x0, x1, x2, sa[j], sb[j], P.kappa, sr, cr, si, ci);
          p2p_pair_mixed(x0, x1, x2, sa[j + G], sb[j + G], P.kappa, sr, cr, si, ci);
        }
        if (j < fill) p2p_pair_mixed(x0, x1, x2, sa[j], sb[j], P.kappa, sr, cr, si, ci);
      } else {
        for (; j + G < fill; j += 2 * G) {
          p2p_pair64(x0, x1, x2, sa[j], sb[j], sc[j], P.kappa, pr, pim);
          p2p_pair64(x0, x1, x2, sa[j + G], sb[j + G], sc[j + G], P.kappa, pr, pim);
        }
        if (j < fill) p2p_pair64(x0, x1, x2, sa[j], sb[j], sc[j], P.kappa, pr, pim);
      }
    }
    if constexpr (MIXED) {
      pr = (double)sr - (double)cr;
      pim = (double)si - (double)ci;
    }
    for (int o = tp; o < 32; o <<= 1) {
      pr += __shfl_xor_sync(0xffffffffu, pr, o);
      pim += __shfl_xor_sync(0xffffffffu, pim, o);
    }
    if (lane < tp) red[warp][lane] = make_double2(pr, pim);
    __syncthreads();
    if (threadIdx.x < nt) {
      double2 a = red[0][threadIdx.x];
      for (int w = 1; w < 4; w++) {
        a.x += red[w][threadIdx.x].x;
        a.y += red[w][threadIdx.x].y;
      }
      if (tpart)
        tpart[it * 32 + threadIdx.x] = a;  // item partial, added per chunk by k_p2p_items
      else
        pnear[f + threadIdx.x] = a;
    }
  }
}

// Item partial sums of the near field into p, per chunk in item order.
__global__ void k_p2p_items(int64_t nchunk, const int32_t* __restrict__ tfirst, const int32_t* __restrict__ tn,
                            const int64_t* __restrict__ chunk_items, const double2* __restrict__ tpart,
                            double2* __restrict__ pnear) {
  const int t = threadIdx.x & 31;
  for (int64_t ch = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); ch < nchunk;
       ch += (int64_t)gridDim.x * (blockDim.x >> 5)) {
    if (t >= tn[ch]) continue;
    double ar = 0., ai = 0.;
    for (int64_t it = chunk_items[ch]; it < chunk_items[ch + 1]; it++) {
      const double2 v = tpart[it * 32 + t];
      ar += v.x;
      ai += v.y;
    }
    double2 o = pnear[tfirst[ch] + t];
    o.x += ar;
    o.y += ai;
    pnear[tfirst[ch] + t] = o;
  }
}

// ----------------------------------------------------- symmetric near field --
// G(x, y) = exp(i k r) / (4 pi r) of one pair (0 for R < 1e-16, P2P.hpp:66),
// with the arithmetic of p2p_pair<false> (FP64) or p2p_pair_mixed (FP32
// after the FP64 r and k r reduction).
// Branch-free: a pair with R < 1e-16 is evaluated at R = 1 and scaled by 0.
__device__ __forceinline__ double2 green64(double dx, double dy, double dz, double kappa) {
  const double R0 = fma(dx, dx, fma(dy, dy, dz * dz));
  const bool skip = R0 < 1.e-16;
  const double R = skip ? 1. : R0;
  const double pi4m1 = skip ? 0. : 1. / (4. * 3.14159265358979323846);
  double y = rsqrt_approx64(R);
  const double hR = 0.5 * R;
  y = y * fma(-hR * y, y, 1.5);
  y = y * fma(-hR * y, y, 1.5);
  const double K = y * pi4m1;
  double sn_, cs_;
  sincos_cw(y * R * kappa, sn_, cs_);
  return make_double2(cs_ * K, sn_ * K);
}
__device__ __forceinline__ float2 green32(double dx, double dy, double dz, double kappa) {
  const double R0 = fma(dx, dx, fma(dy, dy, dz * dz));
  const bool skip = R0 < 1.e-16;
  const double R = skip ? 1. : R0;
  double yd = rsqrt_approx64(R);
  yd = yd * fma(-0.5 * R * yd, yd, 1.5);
  const float y = (float)yd;
  const double theta = R * yd * kappa;
  const double t = fma(theta, 0.31830988618379067154, 6755399441055744.0);  // + 1.5 * 2^52
  const double n = t - 6755399441055744.0;
  const int odd = __double2loint(t) & 1;
  const float x = (float)fma(-n, 3.14159265358979323846, theta);
  const float xx = x * x;
  float ps = fmaf(xx, 1.6059043836821613e-10f, -2.5052108385441720e-08f);
  ps = fmaf(xx, ps, 2.7557319223985893e-06f);
  ps = fmaf(xx, ps, -1.9841269841269841e-04f);
  ps = fmaf(xx, ps, 8.3333333333333333e-03f);
  ps = fmaf(xx, ps, -1.6666666666666667e-01f);
  ps = fmaf(xx, ps, 1.0f);
  float pc = fmaf(xx, 2.0876756987868099e-09f, -2.7557319223985891e-07f);
  pc = fmaf(xx, pc, 2.4801587301587302e-05f);
  pc = fmaf(xx, pc, -1.3888888888888889e-03f);
  pc = fmaf(xx, pc, 4.1666666666666667e-02f);
  pc = fmaf(xx, pc, -0.5f);
  pc = fmaf(xx, pc, 1.0f);
  const float K0 = odd ? -0.0795774715459476679f * y : 0.0795774715459476679f * y;
  const float K = skip ? 0.f : K0;
  return make_float2(pc * K, x * ps * K);
}

// Near field for a block of right-hand sides (the target-side form of
// k_p2p_tiled): per work item, the chunk's targets in lanes (groups of
// tp >= nt lanes), sources streamed through shared memory with RB charges
// each; one evaluation of G(x, y) (green64 / green32) is multiplied into the
// RB right-hand sides r0 .. r0 + RB - 1 of the R in q (q[j R + r]).  Mixed:
// FP32 products summed in FP32 over at most 16 sources per lane, those
// partial sums added in FP64.
// Sums go to pnear[(t) R + r] (item_chunk == nullptr: items are chunks) or
// to tpart[(item 32 + t) R + r] for k_p2p_items_rhs.
template <bool MIXED, int RB>
struct P2PRhsCfg {
  static constexpr int TS = 256;  // sources per tile
  typedef typename std::conditional<MIXED, float2, double2>::type Q;
  static constexpr size_t smem() { return sizeof(double2) * 2 * TS + sizeof(Q) * TS * RB + sizeof(double2) * 4 * 32 * RB; }
};

template <bool MIXED, int RB>
__global__ void __launch_bounds__(128) k_p2p_rhs(DevPlan P, int64_t nitem, const int32_t* __restrict__ order,
                                                 const int32_t* __restrict__ item_chunk,
                                                 const int32_t* __restrict__ tfirst, const int32_t* __restrict__ tn,
                                                 const int64_t* __restrict__ ptr, const int32_t* __restrict__ sfirst,
                                                 const int32_t* __restrict__ sn, const void* __restrict__ qv, int R,
                                                 int r0, double2* __restrict__ pnear, double2* __restrict__ tpart,
                                                 unsigned long long* __restrict__ queue) {
  typedef P2PRhsCfg<MIXED, RB> G;
  constexpr int TS = G::TS;
  typedef typename G::Q Q;
  const Q* q = static_cast<const Q*>(qv);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* sa = reinterpret_cast<double2*>(smem_raw);
  double2* sb = sa + TS;
  Q* sq = reinterpret_cast<Q*>(sb + TS);
  double2* red = reinterpret_cast<double2*>(sq + TS * RB);  // [4][32][RB]
  __shared__ int64_t cur;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) cur = (int64_t)atomicAdd(queue, 1ULL);
    __syncthreads();
    const int64_t k = cur;
    if (k >= nitem) break;
    const int64_t it = order[k];
    const int64_t ch = item_chunk ? item_chunk[it] : it;
    const int f = tfirst[ch], nt = tn[ch];
    int tp = 1;
    while (tp < nt) tp <<= 1;
    const int groups = 32 / tp, GS = 4 * groups;
    const int mt = lane & (tp - 1), gid = warp * groups + lane / tp;
    const int ti = f + min(mt, nt - 1);
    const double x0 = P.T_pos[3 * (int64_t)ti], x1 = P.T_pos[3 * (int64_t)ti + 1], x2 = P.T_pos[3 * (int64_t)ti + 2];
    double2 acc[RB];
#pragma unroll
    for (int b = 0; b < RB; b++) acc[b] = make_double2(0., 0.);
    const int64_t rb = ptr[it], re = ptr[it + 1];
    int64_t r = rb;
    int off = 0;
    while (r < re) {
      int fill = 0;
      __syncthreads();
      while (r < re && fill < TS) {
        const int s0 = sfirst[r], ns = sn[r];
        const int take = min(ns - off, TS - fill);
        for (int t = threadIdx.x; t < take; t += blockDim.x) {
          const int64_t sj = (int64_t)s0 + off + t;
          const double* y = P.S_pos + 3 * sj;
          sa[fill + t] = make_double2(y[0], y[1]);
          sb[fill + t] = make_double2(y[2], 0.);
        }
        for (int t = threadIdx.x; t < take * RB; t += blockDim.x) {
          const int64_t sj = (int64_t)s0 + off + t / RB;
          sq[fill * RB + t] = q[sj * R + r0 + t % RB];
        }
        fill += take;
        off += take;
        if (off == ns) {
          r++;
          off = 0;
        }
      }
      __syncthreads();
      if constexpr (MIXED) {
        // FP32 products summed in FP32 over at most kFlush sources of this
        // lane, then added into the FP64 sums
        constexpr int kFlush = 16;
        for (int j0 = gid; j0 < fill; j0 += kFlush * GS) {
          const int j1 = min(fill, j0 + kFlush * GS);
          float2 fs[RB];
#pragma unroll
          for (int b = 0; b < RB; b++) fs[b] = make_float2(0.f, 0.f);
#pragma unroll 8
          for (int j = j0; j < j1; j += GS) {
            const double2 a = sa[j], bz = sb[j];
            const Q* qj = sq + j * RB;
            const float2 g = green32(x0 - a.x, x1 - a.y, x2 - bz.x, P.kappa);
            if constexpr (RB % 2 == 0) {  // two right-hand sides per 16-byte load
              const float4* q4 = reinterpret_cast<const float4*>(qj);
#pragma unroll
              for (int b = 0; b < RB; b += 2) {
                const float4 qq = q4[b / 2];
                fs[b].x = fmaf(g.x, qq.x, fmaf(-g.y, qq.y, fs[b].x));
                fs[b].y = fmaf(g.x, qq.y, fmaf(g.y, qq.x, fs[b].y));
                fs[b + 1].x = fmaf(g.x, qq.z, fmaf(-g.y, qq.w, fs[b + 1].x));
                fs[b + 1].y = fmaf(g.x, qq.w, fmaf(g.y, qq.z, fs[b + 1].y));
              }
            } else {
#pragma unroll
              for (int b = 0; b < RB; b++) {
                const float2 qq = qj[b];
                fs[b].x = fmaf(g.x, qq.x, fmaf(-g.y, qq.y, fs[b].x));
                fs[b].y = fmaf(g.x, qq.y, fmaf(g.y, qq.x, fs[b].y));
              }
            }
          }
#pragma unroll
          for (int b = 0; b < RB; b++) {
            acc[b].x += (double)fs[b].x;
            acc[b].y += (double)fs[b].y;
          }
        }
      } else {
#pragma unroll 4
        for (int j = gid; j < fill; j += GS) {
          const double2 a = sa[j], bz = sb[j];
          const Q* qj = sq + j * RB;
          const double2 g = green64(x0 - a.x, x1 - a.y, x2 - bz.x, P.kappa);
#pragma unroll
          for (int b = 0; b < RB; b++) {
            const double2 qq = qj[b];
            acc[b].x = fma(g.x, qq.x, fma(-g.y, qq.y, acc[b].x));
            acc[b].y = fma(g.x, qq.y, fma(g.y, qq.x, acc[b].y));
          }
        }
      }
    }
#pragma unroll
    for (int b = 0; b < RB; b++) {
      for (int o = tp; o < 32; o <<= 1) {
        acc[b].x += __shfl_xor_sync(0xffffffffu, acc[b].x, o);
        acc[b].y += __shfl_xor_sync(0xffffffffu, acc[b].y, o);
      }
      if (lane < tp) red[(warp * 32 + lane) * RB + b] = acc[b];
    }
    __syncthreads();
    for (int o = threadIdx.x; o < nt * RB; o += blockDim.x) {
      const int t = o / RB, b = o % RB;
      double2 a = red[t * RB + b];
      for (int w = 1; w < 4; w++) {
        a.x += red[(w * 32 + t) * RB + b].x;
        a.y += red[(w * 32 + t) * RB + b].y;
      }
      if (tpart)
        tpart[(it * 32 + t) * R + r0 + b] = a;
      else
        pnear[(int64_t)(f + t) * R + r0 + b] = a;
    }
  }
}

// Item partial sums of the near field into p for R right-hand sides, per
// chunk in item order (k_p2p_items with R sums per target).
__global__ void k_p2p_items_rhs(int64_t nchunk, const int32_t* __restrict__ tfirst, const int32_t* __restrict__ tn,
                                const int64_t* __restrict__ chunk_items, const double2* __restrict__ tpart, int R,
                                double2* __restrict__ pnear) {
  const int64_t per = 32 * (int64_t)R;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nchunk * per;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ch = w / per;
    const int t = (int)((w % per) / R), rr = (int)(w % R);
    if (t >= tn[ch]) continue;
    double ar = 0., ai = 0.;
    for (int64_t it = chunk_items[ch]; it < chunk_items[ch + 1]; it++) {
      const double2 v = tpart[(it * 32 + t) * R + rr];
      ar += v.x;
      ai += v.y;
    }
    double2* o = pnear + (int64_t)(tfirst[ch] + t) * R + rr;
    double2 v = *o;
    v.x += ar;
    v.y += ai;
    *o = v;
  }
}

// Tree-order R-wide charges from R stacked user-order vectors:
// q[i R + r] = qin[r stride + perm[i]].
// Vectors r >= nvec of a partly filled block get zero charges.
template <typename T>
__global__ void k_gather_rhs(const double2* __restrict__ qin, const int32_t* __restrict__ perm,
                             typename cpx_t<T>::type* __restrict__ q, int64_t n, int64_t stride, int R, int nvec) {
  const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= n * R) return;
  const int64_t i = w / R;
  const int r = (int)(w % R);
  const double2 v = r < nvec ? qin[r * stride + perm[i]] : make_double2(0., 0.);
  typename cpx_t<T>::type o;
  o.x = (T)v.x;
  o.y = (T)v.y;
  q[w] = o;
}

// out[r stride + perm[i]] = pnear[i R + r] + pfar[i R + r].
__global__ void k_scatter_rhs(const double2* __restrict__ pnear, const double2* __restrict__ pfar,
                              const int32_t* __restrict__ perm, double2* __restrict__ out, int64_t n, int64_t stride,
                              int R, int nvec) {
  const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= n * R) return;
  const int64_t i = w / R;
  const int r = (int)(w % R);
  if (r >= nvec) return;
  double2 a = pnear[w], b = pfar[w];
  a.x += b.x;
  a.y += b.y;
  out[r * stride + perm[i]] = a;
}

// tp steps of a symmetric block: lane ls owns one source (y, qj) and meets
// target (ls + step) mod tp; the target's running sum moves one lane down per
// step.  TP = 32 fixes the segment width at compile time.
// Target records in shared memory as two 16-byte arrays, (x, y) and (z, w)
// with w the FP32 charge's bits (mixed path) or unused (FP64 path, the charge
// in tq): one conflict-free 16-byte load from each per step.  Entry j holds
// target j mod tp (j < 64), so step st of lane ls reads entry ls + st without
// wrapping arithmetic.
__device__ __forceinline__ float2 charge_bits(double w) {
  const long long b = __double_as_longlong(w);
  return make_float2(__int_as_float((int)(b & 0xffffffffLL)), __int_as_float((int)(b >> 32)));
}
__device__ __forceinline__ double charge_word(float2 q) {
  return __longlong_as_double(((long long)(unsigned)__float_as_int(q.y) << 32) | (unsigned)__float_as_int(q.x));
}

template <bool MIXED, int TP>
__device__ __forceinline__ void sym_steps(int ls, int tp_rt, double yx, double yy, double yz,
                                          typename std::conditional<MIXED, float2, double2>::type qj,
                                          const double2* trxy, const double2* trzw, const double2* tq,
                                          double kappa,
                                          typename std::conditional<MIXED, float2, double2>::type& accD,
                                          typename std::conditional<MIXED, float2, double2>::type& accT) {
  const int tp = TP ? TP : tp_rt;
  const double2* txy = trxy + ls;
  const double2* tzw = trzw + ls;
  const double2* tql = tq + ls;
#pragma unroll 8
  for (int st = 0; st < tp; st++) {
    const double2 a = txy[st], b = tzw[st];
    if constexpr (MIXED) {
      const float2 g = green32(a.x - yx, a.y - yy, b.x - yz, kappa);
      const float2 qi = charge_bits(b.y);
      accD.x = fmaf(g.x, qj.x, fmaf(-g.y, qj.y, accD.x));
      accD.y = fmaf(g.x, qj.y, fmaf(g.y, qj.x, accD.y));
      accT.x = fmaf(g.x, qi.x, fmaf(-g.y, qi.y, accT.x));
      accT.y = fmaf(g.x, qi.y, fmaf(g.y, qi.x, accT.y));
    } else {
      const double2 g = green64(a.x - yx, a.y - yy, b.x - yz, kappa);
      const double2 qi = tql[st];
      accD.x = fma(g.x, qj.x, fma(-g.y, qj.y, accD.x));
      accD.y = fma(g.x, qj.y, fma(g.y, qj.x, accD.y));
      accT.x = fma(g.x, qi.x, fma(-g.y, qi.y, accT.x));
      accT.y = fma(g.x, qi.y, fma(g.y, qi.x, accT.y));
    }
    accD.x = __shfl_sync(0xffffffffu, accD.x, ls + 1, tp);
    accD.y = __shfl_sync(0xffffffffu, accD.y, ls + 1, tp);
  }
}

// Symmetric blocks of the near field (Plan::sym_*): one CTA (4 warps) per
// work item (part of the sources of one chunk of <= 32 targets), items taken
// from a queue in the host's order of decreasing work.  A warp splits into segments
// of tp = nextpow2(nt) lanes; lane l of a segment owns source l of the
// segment's tp-source sub-tile and, over tp steps, meets every target
// i = (l + step) mod tp.  One evaluation of G feeds both
//   the target's partial  (an accumulator that moves one lane down per step
//                          and ends in lane i), and
//   the source's partial  (lane-local),
// so each mirrored pair of interactions costs one kernel evaluation.  Target
// partials of the item go to tpart (added per chunk by k_p2p_items); source
// partials go to scratch and are added per source leaf by k_p2p_reduce.
template <bool MIXED>
__global__ void __launch_bounds__(128) k_p2p_sym(DevPlan P, int64_t nwork, const int32_t* __restrict__ order,
                                                 const int32_t* __restrict__ item_chunk,
                                                 const int32_t* __restrict__ tfirst, const int32_t* __restrict__ tn,
                                                 const int64_t* __restrict__ ptr, const int32_t* __restrict__ sfirst,
                                                 const int32_t* __restrict__ sn, const int64_t* __restrict__ soff,
                                                 const void* __restrict__ qv, double2* __restrict__ tpart,
                                                 void* __restrict__ scratch, unsigned long long* __restrict__ queue) {
  typedef typename std::conditional<MIXED, float2, double2>::type Q;
  constexpr int RMAX = 128;
  const Q* q = static_cast<const Q*>(qv);
  Q* scr = static_cast<Q*>(scratch);
  __shared__ double2 trxy[64], trzw[64];
  __shared__ double2 tq[64];  // FP64 path: target charges
  __shared__ int32_t rpre[RMAX + 1], rfst[RMAX];
  __shared__ int64_t roff[RMAX];
  __shared__ double2 red[4][32];
  __shared__ int64_t cur;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) cur = (int64_t)atomicAdd(queue, 1ULL);
    __syncthreads();
    const int64_t k = cur;
    if (k >= nwork) break;
    const int64_t it = order[k];
    const int64_t ch = item_chunk[it];
    const int f = tfirst[ch], nt = tn[ch];
    int tp = 4;
    while (tp < nt) tp <<= 1;
    const int ls = lane & (tp - 1);
    if (threadIdx.x < 64) {
      const int j = threadIdx.x, t = j & (tp - 1);
      if (t < nt) {
        const double* x = P.T_pos + 3 * (int64_t)(f + t);
        const Q qt = q[f + t];
        double w = 0.;
        if constexpr (MIXED) {
          w = charge_word(qt);
        } else {
          tq[j] = qt;
        }
        trxy[j] = make_double2(x[0], x[1]);
        trzw[j] = make_double2(x[2], w);
      } else {
        trxy[j] = make_double2(0., 0.);
        trzw[j] = make_double2(0., 0.);
        tq[j] = make_double2(0., 0.);
      }
    }
    float sr = 0.f, cr = 0.f, si = 0.f, ci = 0.f;  // mixed: compensated target sums
    double pr = 0., pim = 0.;                      // FP64 target sums
    const int64_t rb = ptr[it], re = ptr[it + 1];
    for (int64_t r0 = rb; r0 < re; r0 += RMAX) {
      const int nr = (int)min((int64_t)RMAX, re - r0);
      __syncthreads();  // previous batch of ranges (and the target arrays) settled
      for (int m = threadIdx.x; m < nr; m += blockDim.x) {
        rfst[m] = sfirst[r0 + m];
        roff[m] = soff[r0 + m];
        rpre[m + 1] = sn[r0 + m];
      }
      __syncthreads();
      if (warp == 0) {  // inclusive scan of the range lengths
        int carry = 0;
        for (int b0 = 0; b0 < nr; b0 += 32) {
          int v = b0 + lane < nr ? rpre[b0 + lane + 1] : 0;
          for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
          }
          if (b0 + lane < nr) rpre[b0 + lane + 1] = carry + v;
          carry += __shfl_sync(0xffffffffu, v, 31);
        }
        if (lane == 0) rpre[0] = 0;
      }
      __syncthreads();
      const int ntot = rpre[nr];
      for (int base = warp * 32; base < ntot; base += 4 * 32) {
        const int jj = base + lane;
        const bool vj = jj < ntot;
        double yx = 0., yy = 0., yz = 0.;
        Q qj = Q{0, 0};
        int64_t sidx = 0;
        if (vj) {
          int lo = 0, hi = nr - 1;  // last range with rpre <= jj
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (rpre[mid] <= jj) lo = mid; else hi = mid - 1;
          }
          const int o = jj - rpre[lo];
          const int64_t sj = (int64_t)rfst[lo] + o;
          sidx = roff[lo] + o;
          const double* y = P.S_pos + 3 * sj;
          yx = y[0];
          yy = y[1];
          yz = y[2];
          qj = q[sj];
        }
        Q accD = Q{0, 0}, accT = Q{0, 0};
        // no validity tests: padded targets and missing sources carry zero
        // charges, and their target sums are never stored
        if (tp == 32)
          sym_steps<MIXED, 32>(ls, 32, yx, yy, yz, qj, trxy, trzw, tq, P.kappa, accD, accT);
        else
          sym_steps<MIXED, 0>(ls, tp, yx, yy, yz, qj, trxy, trzw, tq, P.kappa, accD, accT);
        if constexpr (MIXED) {
          kahan_add(sr, cr, accD.x);
          kahan_add(si, ci, accD.y);
        } else {
          pr += accD.x;
          pim += accD.y;
        }
        if (vj) scr[sidx] = accT;
      }
    }
    if constexpr (MIXED) {
      pr = (double)sr - (double)cr;
      pim = (double)si - (double)ci;
    }
    for (int o = tp; o < 32; o <<= 1) {  // segments of the warp hold the same targets
      pr += __shfl_xor_sync(0xffffffffu, pr, o);
      pim += __shfl_xor_sync(0xffffffffu, pim, o);
    }
    if (lane < tp) red[warp][lane] = make_double2(pr, pim);
    __syncthreads();
    if (threadIdx.x < nt) {
      double2 a = red[0][threadIdx.x];
      for (int w = 1; w < 4; w++) {
        a.x += red[w][threadIdx.x].x;
        a.y += red[w][threadIdx.x].y;
      }
      tpart[it * 32 + threadIdx.x] = a;
    }
  }
}

// Source-side partial sums of the symmetric blocks, per source leaf in a
// fixed order (Plan::red_*): p_j += sum_k scratch[off_k + (j - first)].
// One CTA per leaf: 4 groups of 64 threads (one particle each) sum
// contiguous quarters of the leaf's rows, row offsets staged in shared
// memory and four rows in flight per thread; the quarters are added in order.
template <bool MIXED>
__global__ void __launch_bounds__(256) k_p2p_reduce(int64_t nleaf, const int32_t* __restrict__ first,
                                                    const int32_t* __restrict__ n, const int64_t* __restrict__ rptr,
                                                    const int64_t* __restrict__ roff, const void* __restrict__ scratch,
                                                    double2* __restrict__ pnear) {
  typedef typename std::conditional<MIXED, float2, double2>::type Q;
  constexpr int RB = 256;  // row offsets staged per round
  const Q* scr = static_cast<const Q*>(scratch);
  __shared__ int64_t so[RB];
  __shared__ double2 part[4][64];
  const int g = threadIdx.x >> 6, jl = threadIdx.x & 63;
  // (leaf, block of 64 particles): leaves of more than 64 particles take
  // several passes
  for (int64_t l = blockIdx.x; l < nleaf; l += gridDim.x)
  for (int j0 = 0; j0 < n[l]; j0 += 64) {
    const int nl = n[l], j = j0 + jl;
    const int64_t kb = rptr[l], ke = rptr[l + 1];
    double ar = 0., ai = 0.;
    __syncthreads();  // the previous pass is done with part[][]
    for (int64_t k0 = kb; k0 < ke; k0 += RB) {
      const int nr = (int)min((int64_t)RB, ke - k0);
      __syncthreads();
      for (int t = threadIdx.x; t < nr; t += blockDim.x) so[t] = roff[k0 + t];
      __syncthreads();
      // group g takes rows [g*nr/4, (g+1)*nr/4) of this round
      const int r0 = g * nr / 4, r1 = (g + 1) * nr / 4;
      if (j < nl) {
        int r = r0;
        for (; r + 4 <= r1; r += 4) {
          const Q v0 = scr[so[r] + j], v1 = scr[so[r + 1] + j], v2 = scr[so[r + 2] + j], v3 = scr[so[r + 3] + j];
          ar += (double)v0.x;
          ai += (double)v0.y;
          ar += (double)v1.x;
          ai += (double)v1.y;
          ar += (double)v2.x;
          ai += (double)v2.y;
          ar += (double)v3.x;
          ai += (double)v3.y;
        }
        for (; r < r1; r++) {
          const Q v = scr[so[r] + j];
          ar += (double)v.x;
          ai += (double)v.y;
        }
      }
    }
    part[g][jl] = make_double2(ar, ai);
    __syncthreads();
    if (g == 0 && j < nl) {
      double2 o = pnear[first[l] + j];
      for (int q = 0; q < 4; q++) {
        o.x += part[q][jl].x;
        o.y += part[q][jl].y;
      }
      pnear[first[l] + j] = o;
    }
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
// twiddles exp(-2 pi i m / P) of every order, computed on the device
__global__ void k_twiddles(double* tw) {
  for (int L = kMinOrder; L <= kMaxOrder; L++) {
    const int P = 2 * L - 1;
    for (int m = threadIdx.x; m < P; m += blockDim.x) {
      double s, c;
      sincospi(-2.0 * m / P, &s, &c);
      tw[2 * (tw_off(L) + m)] = c;
      tw[2 * (tw_off(L) + m) + 1] = s;
    }
  }
}

// Constant tables of the current device: twiddles of every order on first
// use, the interpolation matrices of order L (m2m[0], m2m[1], l2l[0], l2l[1];
// they depend on L only) on first use of L.  Later calls write nothing, so
// kernels of other operators in flight never see a table change.
cudaError_t upload_tables(int L, const double* mats) {
  static std::mutex mu;
  static std::set<std::pair<int, int>> done;  // (device, L); L = 0: twiddles
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (!done.count({dev, 0})) {
    constexpr int n = 2 * tw_off(kMaxOrder + 1);
    double* d = nullptr;
    if ((e = cudaMalloc(&d, n * sizeof(double))) != cudaSuccess) return e;
    k_twiddles<<<1, 32>>>(d);
    std::vector<double> h64(n);
    e = cudaMemcpy(h64.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return e;
    std::vector<float> h32(h64.begin(), h64.end());
    if ((e = cudaMemcpyToSymbol(c_tw64, h64.data(), n * sizeof(double))) != cudaSuccess ||
        (e = cudaMemcpyToSymbol(c_tw32, h32.data(), n * sizeof(float))) != cudaSuccess)
      return e;
    done.insert({dev, 0});
  }
  if (!done.count({dev, L})) {
    const int n = 4 * L * L;
    std::vector<float> m32(mats, mats + n);
    if ((e = cudaMemcpyToSymbol(c_mat64, mats, n * sizeof(double), mat_off(L) * sizeof(double))) != cudaSuccess ||
        (e = cudaMemcpyToSymbol(c_mat32, m32.data(), n * sizeof(float), mat_off(L) * sizeof(float))) != cudaSuccess)
      return e;
    done.insert({dev, L});
  }
  return cudaSuccess;
}

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
  static size_t smem_m2f() { return sizeof(C) * M2FCfg<T, L>::PER_WARP * M2FCfg<T, L>::NW; }
  static size_t smem_m2l() { return sizeof(C) * (PP + L * P * P + L * L * P); }
  template <int RB>
  static size_t smem_m2l_rhs() { return (m2l_rhs_joint<T, L, RB>() ? RB : 1) * smem_m2l(); }
  static cudaError_t setup(const double* mats) {
    cudaError_t e0 = upload_tables(L, mats);
    if (e0 != cudaSuccess) return e0;
    cudaError_t e = cudaFuncSetAttribute(k_m2f<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_m2f());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_m2l<T, L, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_m2l());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_m2l<T, L, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_m2l());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_m2l_pair<T, L, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_m2l());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_m2l_pair<T, L, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_m2l());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_p2m<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)P2MCfg<T, L>::smem(kMaxRhsBlock));
    if (e != cudaSuccess) return e;
    if ((e = rhs_attr<1, 128>()) != cudaSuccess || (e = rhs_attr<2, 128>()) != cudaSuccess ||
        (e = rhs_attr<4, 256>()) != cudaSuccess || (e = rhs_attr<8, 256>()) != cudaSuccess ||
        (e = bulk_attr()) != cudaSuccess)
      return e;
    return cudaSuccess;
  }
  // largest block of right-hand sides per M2L CTA: K x RB <= 24 complex
  // accumulators per thread at 256 threads
  static constexpr int kMaxRB = (PP + 255) / 256 <= 3 ? 8 : ((PP + 255) / 256 <= 6 ? 4 : ((PP + 255) / 256 <= 12 ? 2 : 1));
  template <int RB, int NT>
  static cudaError_t rhs_attr() {
    if (RB > kMaxRB) return cudaSuccess;
    return cudaFuncSetAttribute(k_m2l_rhs<T, L, NT, (RB <= kMaxRB ? RB : 1)>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_m2l_rhs<(RB <= kMaxRB ? RB : 1)>());
  }
  template <int RB, int NT>
  static void m2l_rhs_go(const DevPlan& dp, int64_t t0, int64_t t1, int64_t f0, int64_t f1, int R, const void* F,
                         const void* ptab, void* Lx, unsigned long long* queue, int nsm, cudaStream_t s) {
    constexpr int RBE = RB <= kMaxRB ? RB : 1;
    const int64_t nwork = (t1 - t0) * (R / RBE);
    const int grid = (int)std::min<int64_t>(nwork, (int64_t)nsm * m2l_rhs_ctas<T, NT, RBE>());
    k_m2l_rhs<T, L, NT, RBE><<<grid, NT, smem_m2l_rhs<RBE>(), s>>>(dp, t0, t1, f0, f1, R, (const C*)F, (const C*)ptab,
                                                          (C*)Lx, queue);
  }
  // the shared-memory-staged kernel: FP32, orders 3-6
  static constexpr bool kBulk = std::is_same<T, float>::value && L >= 3 && L <= 6;
  static cudaError_t bulk_attr() {
    if constexpr (kBulk)
      return cudaFuncSetAttribute(k_m2l_bulk<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)M2LBulk<L>::smem());
    return cudaSuccess;
  }
  static bool m2l_bulk(const DevPlan& dp, int64_t t0, int64_t t1, int64_t f0, int64_t f1, int R, const void* F,
                       const void* ptab, void* Lx, unsigned long long* queue, int nsm, int64_t lgroup,
                       cudaStream_t s) {
    if constexpr (kBulk) {
      typedef M2LBulk<L> B;
      if (lgroup <= 0 || lgroup > B::LCAP || R % B::RB) return false;
      const int64_t nwork = (t1 - t0 + B::G - 1) / B::G * (R / B::RB);
      const int grid = (int)std::min<int64_t>(nwork, (int64_t)nsm * B::CTAS);
      k_m2l_bulk<L><<<grid, B::NT, B::smem(), s>>>(dp, t0, t1, f0, f1, R, (const float2*)F, (const float2*)ptab,
                                                   (float2*)Lx, queue);
      return true;
    }
    return false;
  }
  // M2L for R right-hand sides in blocks of rb (1, 2, 4 or 8; a divisor of
  // R, capped by the order's kMaxRB), or staged through shared memory
  static void m2l_rhs(const DevPlan& dp, int64_t t0, int64_t t1, int64_t f0, int64_t f1, int R, int rb,
                      const void* F, const void* ptab, void* Lx, unsigned long long* queue, int nsm,
                      int64_t lgroup, cudaStream_t s) {
    if (t1 <= t0) return;
    cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
    if (m2l_bulk(dp, t0, t1, f0, f1, R, F, ptab, Lx, queue, nsm, lgroup, s)) return;
    if (rb > kMaxRB) rb = kMaxRB;
    while (rb > 1 && R % rb) rb >>= 1;
    if (rb >= 8)
      m2l_rhs_go<8, 256>(dp, t0, t1, f0, f1, R, F, ptab, Lx, queue, nsm, s);
    else if (rb >= 4)
      m2l_rhs_go<4, 256>(dp, t0, t1, f0, f1, R, F, ptab, Lx, queue, nsm, s);
    else if (rb >= 2)
      m2l_rhs_go<2, 128>(dp, t0, t1, f0, f1, R, F, ptab, Lx, queue, nsm, s);
    else
      m2l_rhs_go<1, 128>(dp, t0, t1, f0, f1, R, F, ptab, Lx, queue, nsm, s);
  }
  static void p2m(const DevPlan& dp, const int32_t* leaves, int n, const void* q, const void* sig2, void* M, int R,
                  int d0, int d1, cudaStream_t s) {
    if (n)
      k_p2m<T, L><<<grid_for(n, 1), 128, P2MCfg<T, L>::smem(R), s>>>(dp, leaves, n, (const C*)q, (const C*)sig2,
                                                                     (C*)M, R, d0, d1);
  }
  static void m2m(const DevPlan& dp, int64_t s0, int64_t s1, const void* sig, const void* sig2, void* Mp,
                  const void* Mc, int R, cudaStream_t s) {
    constexpr int NW = kXferWarps;
    if (s1 > s0)
      k_m2m<T, L><<<grid_for(s1 - s0, NW), 32 * NW, 0, s>>>(dp, s0, s1, (const C*)sig, (const C*)sig2, (C*)Mp,
                                                                  (const C*)Mc, R);
  }
  static void l2l(const DevPlan& dp, int64_t s0, int64_t s1, const void* sig, const void* sig2, void* Lc,
                  const void* Lp, int R, int64_t p0, int64_t p1, cudaStream_t s) {
    constexpr int NW = kXferWarps;
    if (s1 > s0)
      k_l2l<T, L><<<grid_for(s1 - s0, NW), 32 * NW, 0, s>>>(dp, s0, s1, (const C*)sig, (const C*)sig2, (C*)Lc,
                                                                  (const C*)Lp, R, p0, p1);
  }
  static void m2f(int64_t n, const void* M, void* F, cudaStream_t s) {
    constexpr int NW = M2FCfg<T, L>::NW;
    if (n) k_m2f<T, L><<<grid_for(n, NW), 32 * NW, smem_m2f(), s>>>(n, (const C*)M, (C*)F);
  }
  static void m2l(const DevPlan& dp, int64_t t0, int64_t t1, int64_t f0, int64_t f1, const void* F,
                  const void* ptab, void* Lx, unsigned long long* queue, int nsm, int nt, int pair,
                  cudaStream_t s) {
    if (t1 <= t0) return;
    cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
    if (nt != 128 && nt != 256) nt = NT;
    if (pair) {
      const int grid = (int)std::min<int64_t>((t1 - t0 + 1) / 2, (int64_t)nsm * (2048 / nt));
      if (nt == 256)
        k_m2l_pair<T, L, 256><<<grid, 256, smem_m2l(), s>>>(dp, t0, t1, f0, f1, (const C*)F, (const C*)ptab, (C*)Lx,
                                                            queue);
      else
        k_m2l_pair<T, L, 128><<<grid, 128, smem_m2l(), s>>>(dp, t0, t1, f0, f1, (const C*)F, (const C*)ptab, (C*)Lx,
                                                            queue);
      return;
    }
    const int grid = (int)std::min<int64_t>(t1 - t0, (int64_t)nsm * (2048 / nt));
    if (nt == 256)
      k_m2l<T, L, 256><<<grid, 256, smem_m2l(), s>>>(dp, t0, t1, f0, f1, (const C*)F, (const C*)ptab, (C*)Lx, queue);
    else
      k_m2l<T, L, 128><<<grid, 128, smem_m2l(), s>>>(dp, t0, t1, f0, f1, (const C*)F, (const C*)ptab, (C*)Lx, queue);
  }
  static void permute(int64_t n, const uint32_t* key, const uint16_t* perm, const void* tables, void* out,
                      cudaStream_t s) {
    if (n) k_permute_tables<T><<<grid_for(n, 1), 256, 0, s>>>(n, PP, key, perm, (const C*)tables, (C*)out);
  }
  static void l2p(const DevPlan& dp, const int32_t* leaves, int n, const void* sig2, const void* Lx, double2* pfar,
                  int R, int d0, int d1, bool accum, cudaStream_t s) {
    if (!n) return;
    if (R == 1)
      k_l2p<T, L, 1><<<grid_for(n, 1), 128, 0, s>>>(dp, leaves, n, (const C*)sig2, (const C*)Lx, pfar, R, d0, d1,
                                                    accum);
    else
      k_l2p<T, L, 4><<<grid_for(n, 1), 128, 0, s>>>(dp, leaves, n, (const C*)sig2, (const C*)Lx, pfar, R, d0, d1,
                                                    accum);
  }
};

template <typename T>
const OpTable* op_table_for(int L);

#define DFB_OPS(T, L)                                                                                     \
  {                                                                                                       \
    Launch<T, L>::setup, Launch<T, L>::p2m, Launch<T, L>::m2m, Launch<T, L>::l2l, Launch<T, L>::m2f,       \
        Launch<T, L>::m2l, Launch<T, L>::m2l_rhs, Launch<T, L>::l2p, Launch<T, L>::permute,                 \
        Launch<T, L>::kMaxRB                                                                              \
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

void launch_p2p(bool fp64, const DevPlan& dp, int64_t nitem, const int32_t* order, const int32_t* item_chunk,
                const int32_t* tfirst, const int32_t* tn, const int64_t* ptr, const int32_t* sfirst, const int32_t* sn,
                const void* q, double2* pnear, double2* tpart, unsigned long long* queue, int nsm, cudaStream_t s) {
  if (!nitem) return;
  cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
  const int grid = (int)std::min<int64_t>(nitem, (int64_t)nsm * 16);
  if (fp64)
    k_p2p_tiled<false><<<grid, 128, 0, s>>>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, pnear,
                                            tpart, queue);
  else
    k_p2p_tiled<true><<<grid, 128, 0, s>>>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, pnear,
                                           tpart, queue);
}

void launch_p2p_items(int64_t nchunk, const int32_t* tfirst, const int32_t* tn, const int64_t* chunk_items,
                      const double2* tpart, double2* pnear, int nsm, cudaStream_t s) {
  if (nchunk <= 0) return;
  const int grid = (int)std::min<int64_t>((nchunk + 3) / 4, (int64_t)nsm * 16);
  k_p2p_items<<<grid, 128, 0, s>>>(nchunk, tfirst, tn, chunk_items, tpart, pnear);
}

void launch_p2p_sym(bool fp64, const DevPlan& dp, int64_t nwork, const int32_t* order, const int32_t* item_chunk,
                    const int32_t* tfirst, const int32_t* tn, const int64_t* ptr, const int32_t* sfirst,
                    const int32_t* sn, const int64_t* soff, const void* q, double2* tpart, void* scratch,
                    unsigned long long* queue, int nsm, int blocks_per_sm, cudaStream_t s) {
  if (nwork <= 0) return;
  cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
  const int grid = (int)std::min<int64_t>(nwork, (int64_t)nsm * std::max(1, std::min(blocks_per_sm, 64)));
  if (fp64)
    k_p2p_sym<false><<<grid, 128, 0, s>>>(dp, nwork, order, item_chunk, tfirst, tn, ptr, sfirst, sn, soff, q, tpart,
                                          scratch, queue);
  else
    k_p2p_sym<true><<<grid, 128, 0, s>>>(dp, nwork, order, item_chunk, tfirst, tn, ptr, sfirst, sn, soff, q, tpart,
                                         scratch, queue);
}

void launch_p2p_reduce(bool fp64, int64_t nleaf, const int32_t* first, const int32_t* n, const int64_t* rptr,
                       const int64_t* roff, const void* scratch, double2* pnear, int nsm, cudaStream_t s) {
  if (nleaf <= 0) return;
  const int grid = (int)std::min<int64_t>(nleaf, (int64_t)nsm * 16);
  if (fp64)
    k_p2p_reduce<false><<<grid, 256, 0, s>>>(nleaf, first, n, rptr, roff, scratch, pnear);
  else
    k_p2p_reduce<true><<<grid, 256, 0, s>>>(nleaf, first, n, rptr, roff, scratch, pnear);
}

cudaError_t setup_rhs_kernels() {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_p2p_rhs<true, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)P2PRhsCfg<true, 8>::smem())) != cudaSuccess ||
      (e = cudaFuncSetAttribute(k_p2p_rhs<false, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)P2PRhsCfg<false, 8>::smem())) != cudaSuccess ||
      (e = cudaFuncSetAttribute(k_p2p_rhs<true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)P2PRhsCfg<true, 4>::smem())) != cudaSuccess ||
      (e = cudaFuncSetAttribute(k_p2p_rhs<false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)P2PRhsCfg<false, 4>::smem())) != cudaSuccess)
    return e;
  return cudaSuccess;
}

template <bool MIXED, int RB>
static void p2p_rhs_go(const DevPlan& dp, int64_t nitem, const int32_t* order, const int32_t* item_chunk,
                       const int32_t* tfirst, const int32_t* tn, const int64_t* ptr, const int32_t* sfirst,
                       const int32_t* sn, const void* q, int R, int r0, double2* pnear, double2* tpart,
                       unsigned long long* queue, int grid, cudaStream_t s) {
  k_p2p_rhs<MIXED, RB><<<grid, 128, P2PRhsCfg<MIXED, RB>::smem(), s>>>(dp, nitem, order, item_chunk, tfirst, tn, ptr,
                                                                       sfirst, sn, q, R, r0, pnear, tpart, queue);
}

void launch_p2p_rhs(bool fp64, const DevPlan& dp, int64_t nitem, const int32_t* order, const int32_t* item_chunk,
                    const int32_t* tfirst, const int32_t* tn, const int64_t* ptr, const int32_t* sfirst,
                    const int32_t* sn, const void* q, int R, double2* pnear, double2* tpart,
                    unsigned long long* queue, int nsm, int blocks_per_sm, cudaStream_t s) {
  if (!nitem) return;
  const int grid = (int)std::min<int64_t>(nitem, (int64_t)nsm * std::max(1, std::min(blocks_per_sm, 64)));
  for (int r0 = 0; r0 < R;) {
    const int left = R - r0;
    const int rb = left >= 8 ? 8 : (left >= 4 ? 4 : 1);
    cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
    if (rb == 8) {
      if (fp64) p2p_rhs_go<false, 8>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, R, r0, pnear, tpart, queue, grid, s);
      else p2p_rhs_go<true, 8>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, R, r0, pnear, tpart, queue, grid, s);
    } else if (rb == 4) {
      if (fp64) p2p_rhs_go<false, 4>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, R, r0, pnear, tpart, queue, grid, s);
      else p2p_rhs_go<true, 4>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, R, r0, pnear, tpart, queue, grid, s);
    } else {
      if (fp64) p2p_rhs_go<false, 1>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, R, r0, pnear, tpart, queue, grid, s);
      else p2p_rhs_go<true, 1>(dp, nitem, order, item_chunk, tfirst, tn, ptr, sfirst, sn, q, R, r0, pnear, tpart, queue, grid, s);
    }
    r0 += rb;
  }
}

void launch_p2p_items_rhs(int64_t nchunk, const int32_t* tfirst, const int32_t* tn, const int64_t* chunk_items,
                          const double2* tpart, int R, double2* pnear, int nsm, cudaStream_t s) {
  if (nchunk <= 0) return;
  const int grid = (int)std::min<int64_t>((nchunk * 32 * R + 255) / 256, (int64_t)nsm * 16);
  k_p2p_items_rhs<<<grid, 256, 0, s>>>(nchunk, tfirst, tn, chunk_items, tpart, R, pnear);
}

void launch_gather_rhs(bool fp64, const double2* qin, const int32_t* perm, void* q, int64_t n, int64_t stride, int R,
                       int nvec, cudaStream_t s) {
  const int g = (int)((n * R + 255) / 256);
  if (fp64)
    k_gather_rhs<double><<<g, 256, 0, s>>>(qin, perm, (double2*)q, n, stride, R, nvec);
  else
    k_gather_rhs<float><<<g, 256, 0, s>>>(qin, perm, (float2*)q, n, stride, R, nvec);
}

void launch_scatter_rhs(const double2* pnear, const double2* pfar, const int32_t* perm, double2* out, int64_t n,
                        int64_t stride, int R, int nvec, cudaStream_t s) {
  k_scatter_rhs<<<(int)((n * R + 255) / 256), 256, 0, s>>>(pnear, pfar, perm, out, n, stride, R, nvec);
}

void launch_direct(int64_t ns, const double* spos, const int32_t* sperm, const double2* qin, int64_t nt,
                   const double* tpos, double kappa, double2* out, cudaStream_t s) {
  if (nt) k_direct<<<grid_for(nt, 8, 148 * 16), 256, 0, s>>>(ns, spos, sperm, qin, nt, tpos, kappa, out);
}

}  // namespace dfb
