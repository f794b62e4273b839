// Host-visible launchers of the matvec kernels (fmm_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace dfb {

// Consecutive target slots per CTA of the shared-memory-staged M2L.
constexpr int kM2LGroup = 4;

// Per-(precision, order) launchers of the expansion phases.  Complex arrays
// are passed untyped; their element type is double2 (FP64) or float2.
struct OpTable {
  // per-order kernel attributes and constant tables; mats = m2m[0], m2m[1],
  // l2l[0], l2l[1] (L*L each, A(k, p) at k + p*L)
  cudaError_t (*setup)(const double* mats);
  // Expansions of R right-hand sides per slot: slot s, right-hand side r at
  // base + (s R + r) * LL (the base may be offset so that a buffer holding a
  // range of slots is addressed by global slot numbers).
  // P2M of the leaves' slots with a direction in [d0, d1) (d0 = INT_MIN,
  // d1 = INT_MAX: every slot); q holds R charges per particle, tree order.
  void (*p2m)(const DevPlan&, const int32_t* leaves, int n, const void* q, const void* sig2, void* M, int R, int d0,
              int d1, cudaStream_t);
  // M2M into parent slots [s0, s1) (bases Mp) from their children (bases Mc)
  void (*m2m)(const DevPlan&, int64_t s0, int64_t s1, const void* sig, const void* sig2, void* Mp, const void* Mc,
              int R, cudaStream_t);
  // L2L into child slots [s0, s1) (bases Lc) from their parent slots in
  // [p0, p1) (bases Lp)
  void (*l2l)(const DevPlan&, int64_t s0, int64_t s1, const void* sig, const void* sig2, void* Lc, const void* Lp,
              int R, int64_t p0, int64_t p1, cudaStream_t);
  void (*m2f)(int64_t n, const void* M, void* F, cudaStream_t);
  // M2L with the inverse DFT fused: adds into L of target slots [t0, t1)
  // nt: threads per CTA (128 or 256; 0 = the order's default); pair != 0:
  // two consecutive target slots per CTA sharing their common sources' loads
  void (*m2l)(const DevPlan&, int64_t t0, int64_t t1, int64_t f0, int64_t f1, const void* F, const void* ptab,
              void* Lx, unsigned long long* queue, int nsm, int nt, int pair, cudaStream_t);
  // The same for R right-hand sides (F: R spectra per source slot of the
  // batch, Lx: base as above), rb of them per CTA sharing each spectrum load.
  // lgroup > 0: the longest list total of kM2LGroup consecutive target
  // slots; the FP32 path at orders 3-6 then stages spectra through shared
  // memory with bulk copies, kM2LGroup target slots per CTA sharing each
  // source's loads (bit-identical results); lgroup <= 0: one target slot per
  // CTA.  F and ptab carry 16 bytes of slack after their last spectrum.
  void (*m2l_rhs)(const DevPlan&, int64_t t0, int64_t t1, int64_t f0, int64_t f1, int R, int rb, const void* F,
                  const void* ptab, void* Lx, unsigned long long* queue, int nsm, int64_t lgroup, cudaStream_t);
  // L2P of the leaves' slots with a direction in [d0, d1) into pfar (R per
  // particle), written (accum = false) or added
  void (*l2p)(const DevPlan&, const int32_t* leaves, int n, const void* sig2, const void* Lx, double2* pfar, int R,
              int d0, int d1, bool accum, cudaStream_t);
  // U_k = tables[key_k >> 6][perm[key_k & 63][:]] for the permuted spectra
  void (*permute)(int64_t n, const uint32_t* key, const uint16_t* perm, const void* tables, void* out,
                  cudaStream_t);
  int max_rb;  // largest right-hand-side block per M2L CTA at this order
};

const OpTable* op_table(int L, bool fp64);

void launch_gather(bool fp64, const double2* qin, const int32_t* perm, void* q, int64_t n, int64_t stride_in,
                   int64_t stride_q, int nrhs, cudaStream_t s);
void launch_scatter(const double2* pnear, const double2* pfar, const int32_t* perm, double2* out, int64_t n,
                    cudaStream_t s);
// Near field (k_p2p_tiled) over work items; `order` lists items by
// decreasing work, `queue` is a device counter the launch resets.  With
// item_chunk == nullptr items are chunks and sums are stored into pnear;
// otherwise item partial sums go to tpart (32 per item) and
// launch_p2p_items adds them per chunk, in item order.
void launch_p2p(bool fp64, const DevPlan& dp, int64_t nitem, const int32_t* order, const int32_t* item_chunk,
                const int32_t* tfirst, const int32_t* tn, const int64_t* ptr, const int32_t* sfirst, const int32_t* sn,
                const void* q, double2* pnear, double2* tpart, unsigned long long* queue, int nsm, cudaStream_t s);
void launch_p2p_items(int64_t nchunk, const int32_t* tfirst, const int32_t* tn, const int64_t* chunk_items,
                      const double2* tpart, double2* pnear, int nsm, cudaStream_t s);
// Symmetric near field: symmetric blocks over items (k_p2p_sym: the target
// side to tpart, the source side to scratch) and the per-leaf reduction of
// the scratch into pnear (k_p2p_reduce).  Scratch holds double2 (fp64) or
// float2 (mixed) partial sums.
// blocks_per_sm: CTAs per SM of the queue-driven launch (grid nsm x it)
void launch_p2p_sym(bool fp64, const DevPlan& dp, int64_t nwork, const int32_t* order, const int32_t* item_chunk,
                    const int32_t* tfirst, const int32_t* tn, const int64_t* ptr, const int32_t* sfirst,
                    const int32_t* sn, const int64_t* soff, const void* q, double2* tpart, void* scratch,
                    unsigned long long* queue, int nsm, int blocks_per_sm, cudaStream_t s);
void launch_p2p_reduce(bool fp64, int64_t nleaf, const int32_t* first, const int32_t* n, const int64_t* rptr,
                       const int64_t* roff, const void* scratch, double2* pnear, int nsm, cudaStream_t s);
// Kernel attributes of the right-hand-side block kernels (call once per
// device, outside stream capture).
cudaError_t setup_rhs_kernels();
// Tensor-core (tcgen05, 3-pass split-TF32) P2M of the mixed-precision path
// (tc_interp.cu): same arguments and results as OpTable::p2m for FP32 data,
// order L.  setup_tc_kernels sets their attributes (once per device).
cudaError_t setup_tc_kernels();
void launch_p2m_tc(int L, const DevPlan& dp, const int32_t* leaves, int n, const void* q, const void* sig2, void* M,
                   int R, int d0, int d1, int nsm, cudaStream_t s);
// The same for L2P (OpTable::l2p arguments); leaves of at most 128 points.
void launch_l2p_tc(int L, const DevPlan& dp, const int32_t* leaves, int n, const void* sig2, const void* Lx,
                   double2* pfar, int R, int d0, int d1, bool accum, int nsm, cudaStream_t s);
// Near field of R right-hand sides (q: R charges per particle, tree order),
// target-side, in passes of up to 8 right-hand sides; sums to pnear[i R + r]
// (item_chunk == nullptr) or to tpart[(item 32 + t) R + r], added per chunk
// by launch_p2p_items_rhs.
void launch_p2p_rhs(bool fp64, const DevPlan& dp, int64_t nitem, const int32_t* order, const int32_t* item_chunk,
                    const int32_t* tfirst, const int32_t* tn, const int64_t* ptr, const int32_t* sfirst,
                    const int32_t* sn, const void* q, int R, double2* pnear, double2* tpart,
                    unsigned long long* queue, int nsm, int blocks_per_sm, cudaStream_t s);
void launch_p2p_items_rhs(int64_t nchunk, const int32_t* tfirst, const int32_t* tn, const int64_t* chunk_items,
                          const double2* tpart, int R, double2* pnear, int nsm, cudaStream_t s);
// q[i R + r] = qin[r stride + perm[i]] (zero for r >= nvec);
// out[r stride + perm[i]] = pnear + pfar (r < nvec)
void launch_gather_rhs(bool fp64, const double2* qin, const int32_t* perm, void* q, int64_t n, int64_t stride, int R,
                       int nvec, cudaStream_t s);
void launch_scatter_rhs(const double2* pnear, const double2* pfar, const int32_t* perm, double2* out, int64_t n,
                        int64_t stride, int R, int nvec, cudaStream_t s);
void launch_direct(int64_t ns, const double* spos, const int32_t* sperm, const double2* qin, int64_t nt,
                   const double* tpos, double kappa, double2* out, cudaStream_t s);

}  // namespace dfb
