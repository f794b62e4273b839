// Leaf interpolation on the 5th-generation tensor cores (tcgen05) for the
// mixed-precision path (P2M here; L2P below, the same scheme with the roles
// of points and expansion entries exchanged): P2M as one GEMM per source leaf,
//   M_{s,r}[l] = conj(sig2_s[l]) sum_j Z[l][j] W[j][(s, r)],
//   W[j][(s, r)] = exp(-i k d_s.(y_j - c)) q_j[r]        (P2M.hpp:114-136),
// with the interpolation matrix Z (LL x n, real, mapOnTrees.hpp:37-83) as the
// A operand and the phased charges of a tile of (slot, right-hand side)
// columns, real and imaginary parts as separate columns, as the B operand.
//
// Arithmetic: 3-pass split TF32 (Z = Z_hi + Z_lo, W = W_hi + W_lo with
// Z_hi, W_hi the TF32 roundings; D = Z_hi W_hi + Z_hi W_lo + Z_lo W_hi,
// FP32 accumulation in tensor memory), about FP32 accuracy.
//
// Execution: one CTA (4 warps) per leaf in turn.  Per column tile (64
// complex columns) and chunk of 32 points, the threads write A and B into
// shared memory in the canonical K-major layout without swizzle, one thread
// issues the MMAs (M = 128 expansion entries per tile, N = 128, K = 8 per
// instruction) and commits them to an mbarrier; after the last chunk each
// warp reads its 32 TMEM lanes (expansion entries) and writes the slots'
// expansions.  Every wait on the mbarrier is bounded: on timeout the kernel
// records an error code, waits once more (bounded) for its MMAs and frees
// its tensor memory.
#include <cstdint>

#include "device_math.cuh"
#include "fmm_kernels.h"
#include "kernels.cuh"
#include "ptx.cuh"

namespace dfb {
namespace {

// ------------------------------------------------------------ PTX wrappers --
// Shared-memory matrix descriptor: K-major, no swizzle (canonical layout
// ((8, n), 2) : ((1, SBO), LBO) in 16-byte units), Blackwell version field.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor: D in FP32, A and B in TF32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {  // one whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // one whole warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 TMEM lanes (this warp's quarter) x 32 consecutive FP32 columns
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// TF32 rounding of an FP32 value (nearest, ties away), low 13 bits zero
__device__ __forceinline__ float tf32r(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// ------------------------------------------------------------------ layout --
constexpr int kKC = 32;        // points per K chunk (4 MMA K-steps)
constexpr int kN = 128;        // B rows per tile = 64 complex (slot, right-hand side) columns
constexpr int kCols = kN / 2;  // complex columns per tile
constexpr uint32_t kWait = 1u << 22;  // mbarrier polls before a wait counts as failed

// K-major tiles of kKC values per row: core matrices of 8 rows x 4 values
// (16 bytes per row, 128 bytes per core matrix), the kKC/4 core matrices of
// an 8-row group consecutive (LBO = 128 B), row groups after each other
// (SBO = kKC/4 * 128 B); element (row, k) at byte
//   ((row / 8) * (kKC / 4) + k / 4) * 128 + (row % 8) * 16 + (k % 4) * 4,
// so core matrix cm = (row / 8) * (kKC / 4) + k / 4 holds 32 consecutive
// floats, lane (row % 8) * 4 + k % 4 of a warp writing it.  An MMA K-step ks
// starts at byte ks * 256.
constexpr uint32_t kLBO = 128, kSBO = (kKC / 4) * 128;

template <int L>
struct P2MTc {
  static constexpr int LL = L * L * L;
  static constexpr int MT = (LL + 127) / 128;  // M tiles of 128 expansion entries
  static constexpr uint32_t TCOLS = MT * kN <= 128 ? 128u : (MT * kN <= 256 ? 256u : 512u);
  static constexpr size_t A_BYTES = (size_t)MT * 128 * kKC * 4;  // one of hi / lo
  static constexpr size_t B_BYTES = (size_t)kN * kKC * 4;
  // A hi, A lo, B hi, B lo (1024-byte aligned), basis values, point offsets,
  // phases, charges (R per point)
  static size_t smem(int R) {
    return 1024 + 2 * A_BYTES + 2 * B_BYTES + sizeof(float) * kKC * 3 * L + sizeof(double) * kKC * 3 +
           sizeof(float2) * kKC * kCols + sizeof(float2) * (size_t)kKC * R;
  }
};

}  // namespace

// P2M of the leaves' slots with a direction in [d0, d1) for R right-hand
// sides (q[j R + r], M + (s R + r) LL), FP32 storage, 3-pass split-TF32
// tensor-core GEMMs.  err receives 3 if a tensor-core wait timed out.
template <int L>
__global__ void __launch_bounds__(128, 1) k_p2m_tc(DevPlan P, const int32_t* __restrict__ leaves, int nleaves,
                                                   const float2* __restrict__ q, const float2* __restrict__ sig2,
                                                   float2* __restrict__ M, int R, int d0, int d1) {
  typedef P2MTc<L> G;
  constexpr int LL = G::LL, MT = G::MT;
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_sh;
  __shared__ int fail;
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  float* Ahi = reinterpret_cast<float*>(base);
  float* Alo = Ahi + G::A_BYTES / 4;
  float* Bhi = Alo + G::A_BYTES / 4;
  float* Blo = Bhi + G::B_BYTES / 4;
  float* Bs = Blo + G::B_BYTES / 4;                        // kKC x 3 x L
  double* yc = reinterpret_cast<double*>(Bs + kKC * 3 * L);  // kKC x 3
  float2* E = reinterpret_cast<float2*>(yc + kKC * 3);     // kKC x kCols
  float2* qs = E + kKC * kCols;                            // kKC x R
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tmem_alloc(&tmem_sh, G::TCOLS);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    fail = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;
  const uint32_t aHi = smem_u32(Ahi), aLo = smem_u32(Alo), bHi = smem_u32(Bhi), bLo = smem_u32(Blo);
  uint32_t parity = 0;
  const int ST = R <= kCols ? kCols / R : 1;  // slots per column tile
  for (int li = blockIdx.x; li < nleaves; li += gridDim.x) {
    const int c = leaves[li];
    int64_t sb, se;
    dir_range(P.S_cptr, P.S_cdir, c, d0, d1, &sb, &se);
    const int nslots = (int)(se - sb);
    if (nslots == 0) continue;
    const int n = P.S_nprt[c], f = P.S_first[c];
    const double4 ct = P.S_ctr[c];
    const int lv = P.S_lvl[c];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const double* dirs = P.dirs + P.dir_off[h] * 3;
    const float2* s2 = sig2 + P.sig_off[h];
    const int nchunk = (n + kKC - 1) / kKC;
    for (int s0 = 0; s0 < nslots; s0 += ST) {
      const int ns = min(ST, nslots - s0);
      for (int ch = 0; ch < nchunk; ch++) {
        const int p0 = ch * kKC, np = min(kKC, n - p0);
        // the chunk's points: offsets from the centre, basis values, charges
        for (int o = tid; o < kKC * 3; o += blockDim.x) {
          const int p = o / 3, k = o % 3;
          const double x = p < np ? P.S_pos[3 * (int64_t)(f + p0 + p) + k] - (&ct.x)[k] : 0.;
          yc[o] = x;
          float b[L];
          lagrange_all<L, float>((float)x, (float)ct.w, b);
#pragma unroll
          for (int l = 0; l < L; l++) Bs[o * L + l] = p < np ? b[l] : 0.f;
        }
        for (int o = tid; o < kKC * R; o += blockDim.x) {
          const int p = o / R;
          qs[o] = p < np ? q[(int64_t)(f + p0 + p) * R + o % R] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        // A = Z: rows = expansion entries, K = points (rebuilt when the
        // chunk changes)
        if (nchunk > 1 || s0 == 0) {
          // one 8 x 4 core matrix per warp and store: 32 distinct banks
          for (int cm = warp; cm < MT * 128; cm += 4) {  // (M tile, row group, k block)
            const int row = (cm >> 3) * 8 + (lane >> 2), k = (cm & 7) * 4 + (lane & 3);
            float z = 0.f;
            if (row < LL && k < np) {
              const int i0 = row / (L * L), i1 = (row / L) % L, i2 = row % L;
              z = Bs[(k * 3 + 0) * L + i0] * Bs[(k * 3 + 1) * L + i1] * Bs[(k * 3 + 2) * L + i2];
            }
            const float hi = tf32r(z);
            Ahi[cm * 32 + lane] = hi;
            Alo[cm * 32 + lane] = tf32r(z - hi);
          }
        }
        // phases of the tile's slots at the chunk's points
        for (int o = tid; o < kKC * ns; o += blockDim.x) {
          const int p = o / ns, sl = o % ns;
          float2 e = make_float2(1.f, 0.f);
          if (hf && p < np) {
            const double* dv = dirs + 3 * P.S_cdir[sb + s0 + sl];
            const double dp = dv[0] * yc[3 * p] + dv[1] * yc[3 * p + 1] + dv[2] * yc[3 * p + 2];
            e = expi<float2>(-P.kappa * dp);
          }
          E[p * kCols + sl] = e;
        }
        __syncthreads();
        // B = W: rows = 2 (slot R + r) + (0 real, 1 imaginary), K = points
        for (int cm = warp; cm < kN / 8 * (kKC / 4); cm += 4) {  // (row group, k block)
          const int row = (cm >> 3) * 8 + (lane >> 2), k = (cm & 7) * 4 + (lane & 3);
          const int cp = row >> 1, sl = cp / R, r = cp % R;
          float w = 0.f;
          if (sl < ns && k < np) {
            const float2 e = E[k * kCols + sl], qq = qs[k * R + r];
            w = (row & 1) ? e.x * qq.y + e.y * qq.x : e.x * qq.x - e.y * qq.y;
          }
          const float hi = tf32r(w);
          Bhi[cm * 32 + lane] = hi;
          Blo[cm * 32 + lane] = tf32r(w - hi);
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
          tc_fence_after();
          constexpr uint32_t idesc = idesc_tf32(128, kN);
#pragma unroll
          for (int mt = 0; mt < MT; mt++) {
            const uint32_t d = tmem + (uint32_t)(mt * kN);
#pragma unroll
            for (int ks = 0; ks < kKC / 8; ks++) {
              const uint32_t ao = (uint32_t)(mt * 128 * kKC * 4 + ks * 256), bo = (uint32_t)(ks * 256);
              const uint64_t ah = sdesc(aHi + ao, kLBO, kSBO), al = sdesc(aLo + ao, kLBO, kSBO);
              const uint64_t bh = sdesc(bHi + bo, kLBO, kSBO), bl = sdesc(bLo + bo, kLBO, kSBO);
              mma_tf32(d, ah, bh, idesc, (ch > 0 || ks > 0) ? 1u : 0u);
              mma_tf32(d, ah, bl, idesc, 1u);
              mma_tf32(d, al, bh, idesc, 1u);
            }
          }
          mma_commit(&mbar);
        }
        // the MMAs read A and B: wait for them before the next chunk
        if (!mbar_wait(&mbar, parity, kWait)) atomicExch(&fail, 1);
        parity ^= 1u;
        __syncthreads();
        if (fail) break;
      }
      if (fail) break;
      tc_fence_after();
      // epilogue: warp w holds expansion entries 32 w .. 32 w + 31 of each M tile
#pragma unroll
      for (int mt = 0; mt < MT; mt++) {
        const int l = mt * 128 + warp * 32 + lane;
#pragma unroll
        for (int cb = 0; cb < kN / 32; cb++) {
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * kN + cb * 32), v);
#pragma unroll
          for (int t = 0; t < 16; t++) {
            const int cp = cb * 16 + t, sl = cp / R, r = cp % R;
            if (sl < ns && l < LL) {
              const int slot = P.S_cslot[sb + s0 + sl];
              float2 a = make_float2(v[2 * t], v[2 * t + 1]);
              if (hf) a = cmulc(s2[(int64_t)P.S_cdir[sb + s0 + sl] * LL + l], a);
              M[((int64_t)slot * R + r) * LL + l] = a;
            }
          }
        }
      }
      tc_fence_before();
      __syncthreads();
    }
    if (fail) break;
  }
  if (fail) {
    if (tid == 0) atomicExch(P.err, 3);
    // the last commit may still be pending: wait for it (bounded) before
    // the tensor memory is released
    mbar_wait(&mbar, parity ^ 1u, kWait);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, G::TCOLS);
}

// L2P of the leaves' slots with a direction in [d0, d1) for R right-hand
// sides (Lx + (s R + r) LL) into pfar (R potentials per particle, added):
//   p_r(x_j) += sum_s exp(i k d_s.(x_j - c)) sum_l Z[j][l] sig2_s[l] L_{s,r}[l]
// (L2P.hpp:122-173) as D = Z^T X per target leaf: A = Z^T (rows = the leaf's
// points, <= 128; K = expansion entries in chunks of 32), B = X (rows = real
// and imaginary parts of the tile's (slot, right-hand side) columns).  The
// epilogue multiplies each column pair by the point's phase for that slot
// and sums over the slots into FP64 accumulators, RC <= 8 right-hand sides
// at a time (a tile is 64 / RC slots x RC right-hand sides).
template <int L>
struct L2PTc {
  static constexpr int LL = L * L * L;
  static constexpr int KT = (LL + kKC - 1) / kKC;  // K chunks of 32 expansion entries
  static constexpr size_t A_BYTES = (size_t)128 * kKC * 4;
  static constexpr size_t B_BYTES = (size_t)kN * kKC * 4;
  // A hi, A lo, B hi, B lo (1024-byte aligned), basis values (128 x 3 x L),
  // staged expansions (kCols x (kKC + 1) complex)
  static size_t smem() {
    return 1024 + 2 * A_BYTES + 2 * B_BYTES + sizeof(float) * 128 * 3 * L + sizeof(float2) * kCols * (kKC + 1);
  }
};

template <int L>
__global__ void __launch_bounds__(128, 1) k_l2p_tc(DevPlan P, const int32_t* __restrict__ leaves, int nleaves,
                                                   const float2* __restrict__ sig2, const float2* __restrict__ Lx,
                                                   double2* __restrict__ pfar, int R, int d0, int d1, bool accum) {
  typedef L2PTc<L> G;
  constexpr int LL = G::LL, KT = G::KT;
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_sh;
  __shared__ int fail;
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  float* Ahi = reinterpret_cast<float*>(base);
  float* Alo = Ahi + G::A_BYTES / 4;
  float* Bhi = Alo + G::A_BYTES / 4;
  float* Blo = Bhi + G::B_BYTES / 4;
  float* Bs = Blo + G::B_BYTES / 4;  // 128 points x 3 x L
  float2* Xs = reinterpret_cast<float2*>(Bs + 128 * 3 * L);  // kCols x (kKC + 1)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tmem_alloc(&tmem_sh, 128);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    fail = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;
  const uint32_t aHi = smem_u32(Ahi), aLo = smem_u32(Alo), bHi = smem_u32(Bhi), bLo = smem_u32(Blo);
  uint32_t parity = 0;
  const int RC = R < 8 ? R : 8;  // right-hand sides per tile (and FP64 accumulators per thread)
  const int ST = kCols / RC;     // slots per tile
  const int j = warp * 32 + lane;  // this thread's point (TMEM lane)
  for (int li = blockIdx.x; li < nleaves; li += gridDim.x) {
    const int c = leaves[li];
    int64_t sb, se;
    dir_range(P.T_cptr, P.T_cdir, c, d0, d1, &sb, &se);
    const int nslots = (int)(se - sb);
    if (nslots == 0) continue;
    const int n = min(P.T_nprt[c], 128), f = P.T_first[c];
    const double4 ct = P.T_ctr[c];
    const int lv = P.T_lvl[c];
    const bool hf = P.ishf[lv] != 0;
    const int h = P.hfstage[lv];
    const double* dirs = P.dirs + P.dir_off[h] * 3;
    const float2* s2 = sig2 + P.sig_off[h];
    // the leaf's points: basis values in shared memory, offsets in registers
    __syncthreads();
    double xr[3] = {0., 0., 0.};
    for (int o = tid; o < 128 * 3; o += blockDim.x) {
      const int p = o / 3, k = o % 3;
      const double x = p < n ? P.T_pos[3 * (int64_t)(f + p) + k] - (&ct.x)[k] : 0.;
      float b[L];
      lagrange_all<L, float>((float)x, (float)ct.w, b);
#pragma unroll
      for (int l = 0; l < L; l++) Bs[o * L + l] = p < n ? b[l] : 0.f;
    }
    if (j < n)
      for (int k = 0; k < 3; k++) xr[k] = P.T_pos[3 * (int64_t)(f + j) + k] - (&ct.x)[k];
    for (int r0 = 0; r0 < R; r0 += RC) {
      const int nr = min(RC, R - r0);
      double2 acc[8];
#pragma unroll
      for (int u = 0; u < 8; u++) acc[u] = make_double2(0., 0.);
      for (int s0 = 0; s0 < nslots; s0 += ST) {
        const int ns = min(ST, nslots - s0);
        for (int kc = 0; kc < KT; kc++) {
          const int l0 = kc * kKC;
          __syncthreads();  // Bs written; the previous chunk's MMAs are done (waited below)
          // A = Z^T: rows = points, K = expansion entries l0 .. l0 + 31
          for (int cm = warp; cm < 128 / 8 * (kKC / 4); cm += 4) {  // (row group, k block)
            const int p = (cm >> 3) * 8 + (lane >> 2), k = (cm & 7) * 4 + (lane & 3), l = l0 + k;
            float z = 0.f;
            if (p < n && l < LL) {
              const int i0 = l / (L * L), i1 = (l / L) % L, i2 = l % L;
              z = Bs[(p * 3 + 0) * L + i0] * Bs[(p * 3 + 1) * L + i1] * Bs[(p * 3 + 2) * L + i2];
            }
            const float hi = tf32r(z);
            Ahi[cm * 32 + lane] = hi;
            Alo[cm * 32 + lane] = tf32r(z - hi);
          }
          // B = X: rows = 2 (slot RC + r) + part, K = expansion entries
          // the tile's expansions, read along l (coalesced), scaled by the
          // signatures, staged in Xs (rows padded to 33 entries)
          for (int o = tid; o < kCols * kKC; o += blockDim.x) {
            const int cp = o / kKC, k = o % kKC, l = l0 + k;
            const int sl = cp / RC, r = cp % RC;
            float2 x = make_float2(0.f, 0.f);
            if (sl < ns && r < nr && l < LL) {
              const int64_t js = sb + s0 + sl;
              x = Lx[((int64_t)P.T_cslot[js] * R + r0 + r) * LL + l];
              if (hf) x = cmul(s2[(int64_t)P.T_cdir[js] * LL + l], x);
            }
            Xs[cp * (kKC + 1) + k] = x;
          }
          __syncthreads();
          for (int cm = warp; cm < kN / 8 * (kKC / 4); cm += 4) {  // (row group, k block)
            const int row = (cm >> 3) * 8 + (lane >> 2), k = (cm & 7) * 4 + (lane & 3);
            const float2 x = Xs[(row >> 1) * (kKC + 1) + k];
            const float w = (row & 1) ? x.y : x.x;
            const float hi = tf32r(w);
            Bhi[cm * 32 + lane] = hi;
            Blo[cm * 32 + lane] = tf32r(w - hi);
          }
          fence_async_smem();
          __syncthreads();
          if (tid == 0) {
            tc_fence_after();
            constexpr uint32_t idesc = idesc_tf32(128, kN);
#pragma unroll
            for (int ks = 0; ks < kKC / 8; ks++) {
              const uint32_t o = (uint32_t)(ks * 256);
              const uint64_t ah = sdesc(aHi + o, kLBO, kSBO), al = sdesc(aLo + o, kLBO, kSBO);
              const uint64_t bh = sdesc(bHi + o, kLBO, kSBO), bl = sdesc(bLo + o, kLBO, kSBO);
              mma_tf32(tmem, ah, bh, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
              mma_tf32(tmem, ah, bl, idesc, 1u);
              mma_tf32(tmem, al, bh, idesc, 1u);
            }
            mma_commit(&mbar);
          }
          if (!mbar_wait(&mbar, parity, kWait)) atomicExch(&fail, 1);
          parity ^= 1u;
          __syncthreads();
          if (fail) break;
        }
        if (fail) break;
        tc_fence_after();
        // epilogue: this thread's point, the tile's column pairs times the
        // point's phase for each slot, summed over the slots
#pragma unroll
        for (int cb = 0; cb < kN / 32; cb++) {
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 32), v);
          int last = -1;
          float2 ph = make_float2(1.f, 0.f);
#pragma unroll
          for (int t = 0; t < 16; t++) {
            const int cp = cb * 16 + t, sl = cp / RC, r = cp % RC;
            if (sl < ns && r < nr && j < n) {
              if (hf && sl != last) {
                const double* dv = dirs + 3 * P.T_cdir[sb + s0 + sl];
                ph = expi<float2>(P.kappa * (dv[0] * xr[0] + dv[1] * xr[1] + dv[2] * xr[2]));
                last = sl;
              }
              const float2 val = hf ? cmul(make_float2(v[2 * t], v[2 * t + 1]), ph) : make_float2(v[2 * t], v[2 * t + 1]);
#pragma unroll
              for (int u = 0; u < 8; u++)
                if (u == r) {
                  acc[u].x += (double)val.x;
                  acc[u].y += (double)val.y;
                }
            }
          }
        }
        tc_fence_before();
      }
      if (fail) break;
      if (j < n) {
        for (int u = 0; u < nr; u++) {
          double2* o = pfar + (int64_t)(f + j) * R + r0 + u;
          double2 t = acc[u];
          if (accum) {
            t.x += o->x;
            t.y += o->y;
          }
          *o = t;
        }
      }
    }
    if (fail) break;
  }
  if (fail) {
    if (tid == 0) atomicExch(P.err, 3);
    mbar_wait(&mbar, parity ^ 1u, kWait);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 128);
}

template <int L>
static cudaError_t l2p_tc_setup() {
  return cudaFuncSetAttribute(k_l2p_tc<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L2PTc<L>::smem());
}

template <int L>
static void l2p_tc_go(const DevPlan& dp, const int32_t* leaves, int n, const void* sig2, const void* Lx,
                      double2* pfar, int R, int d0, int d1, bool accum, int nsm, cudaStream_t s) {
  const int grid = (int)std::min<int64_t>(n, (int64_t)nsm * 2);
  k_l2p_tc<L><<<grid, 128, L2PTc<L>::smem(), s>>>(dp, leaves, n, (const float2*)sig2, (const float2*)Lx, pfar, R,
                                                    d0, d1, accum);
}

void launch_l2p_tc(int L, const DevPlan& dp, const int32_t* leaves, int n, const void* sig2, const void* Lx,
                   double2* pfar, int R, int d0, int d1, bool accum, int nsm, cudaStream_t s) {
  if (n <= 0) return;
  switch (L) {
    case 2: l2p_tc_go<2>(dp, leaves, n, sig2, Lx, pfar, R, d0, d1, accum, nsm, s); break;
    case 3: l2p_tc_go<3>(dp, leaves, n, sig2, Lx, pfar, R, d0, d1, accum, nsm, s); break;
    case 4: l2p_tc_go<4>(dp, leaves, n, sig2, Lx, pfar, R, d0, d1, accum, nsm, s); break;
    case 5: l2p_tc_go<5>(dp, leaves, n, sig2, Lx, pfar, R, d0, d1, accum, nsm, s); break;
    case 6: l2p_tc_go<6>(dp, leaves, n, sig2, Lx, pfar, R, d0, d1, accum, nsm, s); break;
    case 7: l2p_tc_go<7>(dp, leaves, n, sig2, Lx, pfar, R, d0, d1, accum, nsm, s); break;
    case 8: l2p_tc_go<8>(dp, leaves, n, sig2, Lx, pfar, R, d0, d1, accum, nsm, s); break;
    default: break;
  }
}

template <int L>
static cudaError_t p2m_tc_setup() {
  return cudaFuncSetAttribute(k_p2m_tc<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)P2MTc<L>::smem(kMaxRhsBlock));
}

cudaError_t setup_tc_kernels() {
  cudaError_t e;
  if ((e = p2m_tc_setup<2>()) != cudaSuccess || (e = p2m_tc_setup<3>()) != cudaSuccess ||
      (e = p2m_tc_setup<4>()) != cudaSuccess || (e = p2m_tc_setup<5>()) != cudaSuccess ||
      (e = p2m_tc_setup<6>()) != cudaSuccess || (e = p2m_tc_setup<7>()) != cudaSuccess ||
      (e = p2m_tc_setup<8>()) != cudaSuccess)
    return e;
  if ((e = l2p_tc_setup<2>()) != cudaSuccess || (e = l2p_tc_setup<3>()) != cudaSuccess ||
      (e = l2p_tc_setup<4>()) != cudaSuccess || (e = l2p_tc_setup<5>()) != cudaSuccess ||
      (e = l2p_tc_setup<6>()) != cudaSuccess || (e = l2p_tc_setup<7>()) != cudaSuccess ||
      (e = l2p_tc_setup<8>()) != cudaSuccess)
    return e;
  return cudaSuccess;
}

template <int L>
static void p2m_tc_go(const DevPlan& dp, const int32_t* leaves, int n, const void* q, const void* sig2, void* M,
                      int R, int d0, int d1, int nsm, cudaStream_t s) {
  const size_t sm = P2MTc<L>::smem(R);
  const int per_sm = sm <= 110 * 1024 ? 2 : 1;
  const int grid = (int)std::min<int64_t>(n, (int64_t)nsm * per_sm);
  k_p2m_tc<L><<<grid, 128, sm, s>>>(dp, leaves, n, (const float2*)q, (const float2*)sig2, (float2*)M, R, d0, d1);
}

void launch_p2m_tc(int L, const DevPlan& dp, const int32_t* leaves, int n, const void* q, const void* sig2, void* M,
                   int R, int d0, int d1, int nsm, cudaStream_t s) {
  if (n <= 0) return;
  switch (L) {
    case 2: p2m_tc_go<2>(dp, leaves, n, q, sig2, M, R, d0, d1, nsm, s); break;
    case 3: p2m_tc_go<3>(dp, leaves, n, q, sig2, M, R, d0, d1, nsm, s); break;
    case 4: p2m_tc_go<4>(dp, leaves, n, q, sig2, M, R, d0, d1, nsm, s); break;
    case 5: p2m_tc_go<5>(dp, leaves, n, q, sig2, M, R, d0, d1, nsm, s); break;
    case 6: p2m_tc_go<6>(dp, leaves, n, q, sig2, M, R, d0, d1, nsm, s); break;
    case 7: p2m_tc_go<7>(dp, leaves, n, q, sig2, M, R, d0, d1, nsm, s); break;
    case 8: p2m_tc_go<8>(dp, leaves, n, q, sig2, M, R, d0, d1, nsm, s); break;
    default: break;
  }
}

}  // namespace dfb
