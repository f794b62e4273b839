/*
 * defmm_b200 -- C ABI of a B200 (sm_100a) implementation of defmm's
 * directional equispaced-interpolation FMM matvec for the Helmholtz kernel
 * G(x, y) = exp(i k |x - y|) / (4 pi |x - y|)  (pairs with |x - y|^2 < 1e-16
 * contribute nothing, as in the reference's P2P.hpp:66).
 *
 * The entry points replace the public interface of IChollet/defmm's
 * `defmm::IBFMM_Mat<3>` (include/interface.hpp:46-224); each declaration cites
 * the member it replaces.  Differences from the reference, by design:
 *   - errors are returned as negative status codes (the reference prints and
 *     calls exit(1)); defmm_last_error() gives the message;
 *   - every defmm_gemv is correct (the reference's gemv never clears its
 *     non-leaf expansions, interface.hpp:159, so only its first call is);
 *   - handles are independent (the reference keeps process-global state).
 * Complex vectors are interleaved (re, im) doubles, indexed in the user's
 * particle order, like the reference's Vecc (std::complex<double>).
 * A handle is not thread-safe; different handles may be used concurrently.
 */
#ifndef DEFMM_B200_H
#define DEFMM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct defmm_handle defmm_handle;

/* Status codes. */
#define DEFMM_OK 0
#define DEFMM_ERR_ARG (-1)        /* invalid argument or call order          */
#define DEFMM_ERR_DEPTH (-2)      /* coincident points: tree never terminates */
#define DEFMM_ERR_SHALLOW (-3)    /* no level admits far-field (M2L) work     */
#define DEFMM_ERR_CUDA (-4)       /* CUDA runtime error / no device           */
#define DEFMM_ERR_MEMORY (-5)     /* device memory exhausted                  */
#define DEFMM_ERR_IO (-6)         /* INP file unreadable or short             */

/* Arithmetic of the matvec. */
#define DEFMM_PRECISION_FP64 0   /* plain FP64, the drop-in for the reference  */
#define DEFMM_PRECISION_MIXED 1  /* FP32 bulk arithmetic, FP64 phase reduction */

/* Number of visible CUDA devices (0 when there is none or no driver). */
int defmm_device_count(void);

/* IBFMM_Mat<3>::IBFMM_Mat() (interface.hpp:57). */
defmm_handle* defmm_create(void);
/* ~IBFMM_Mat: releases host and device memory. */
void defmm_destroy(defmm_handle* h);
/* Message of the last failing call on this handle ("" if none). */
const char* defmm_last_error(const defmm_handle* h);

/* IBFMM_Mat<3>::addSourceParticle(flt part[3]) (interface.hpp:59-67). */
int defmm_add_source_particle(defmm_handle* h, const double xyz[3]);
/* IBFMM_Mat<3>::addTargetParticle(flt part[3]) (interface.hpp:69-77). */
int defmm_add_target_particle(defmm_handle* h, const double xyz[3]);
/* Bulk forms of the two calls above: n points, xyz interleaved. */
int defmm_add_sources(defmm_handle* h, const double* xyz, int64_t n);
int defmm_add_targets(defmm_handle* h, const double* xyz, int64_t n);
/* IBFMM_Mat<3>::addSourceParticlesINP / addTargetParticlesINP
 * (interface.hpp:79-98): read `nparts` lines "x y z" from an INP file.
 * which = 0: sources, 1: targets.  Unlike the reference, a short or missing
 * file is an error (DEFMM_ERR_IO) instead of silently reading zeros. */
int defmm_load_inp(defmm_handle* h, const char* path, int64_t nparts, int which);

/* IBFMM_Mat<3>::prcmpt(int L, int Ncrit, flt kappa, int lvMAX = -1)
 * (interface.hpp:100-151): build both octrees (leaf = fewer than Ncrit
 * particles, or fixed depth lvMAX when lvMAX >= 0), the frequency regime,
 * cones, interaction lists, expansion slots and transfer spectra.  With a
 * GPU present (defmm_set_plan_device) the octrees' particle ordering (octant
 * codes, counts and a stable radix sort per level), the level walk (dual
 * traversal, cones, effective directions, slots, far entries), the M2M/L2L
 * transfer lists, the per-cell slot lists and the near-field work lists run
 * there (and the transfer spectra and signatures at upload), the cells on the
 * host; the results are the host build's, bit for bit.  2 <= L <= 8. */
int defmm_prcmpt(defmm_handle* h, int L, int Ncrit, double kappa, int lvMAX);

/* Copy the plan to the current CUDA device (done by the first gemv when not
 * called explicitly; without a GPU prcmpt runs entirely on the host, so the
 * plan can be inspected without one). */
int defmm_upload(defmm_handle* h);

/* Select the matvec arithmetic (DEFMM_PRECISION_*); default FP64.
 * May be called before or after prcmpt. */
int defmm_set_precision(defmm_handle* h, int mode);

/* friend gemv(IBFMM_Mat&, Vecc& In, Vecc& Out) (interface.hpp:153-170):
 * Out = A * In for host vectors; In has n_sources complex entries, Out
 * n_targets, both in user order.  Blocks until Out is written. */
int defmm_gemv(defmm_handle* h, const double* in, double* out);

/* Device-resident form: d_in / d_out are device pointers to nrhs stacked
 * complex vectors (rhs-major, each in user order).  Runs on `stream`
 * (a cudaStream_t; NULL = the handle's own stream) without synchronising.
 * One right-hand side runs on the resident layout (every expansion on the
 * device, the matvec replayed from a captured graph) when it fits, else on
 * the grouped layout below.  nrhs > 1 runs in passes of up to
 * defmm_set_blocking's rhs_block right-hand sides over the grouped layout:
 * the HF levels' expansions split into direction groups (one group's M and
 * L on the device at a time), and every pass evaluates each near-field
 * kernel value, transfer-spectrum entry and plane-wave phase once for all
 * its right-hand sides. */
int defmm_gemv_device(defmm_handle* h, const void* d_in, void* d_out,
                      int64_t nrhs, void* stream);

/* No counterpart in the reference.  rhs_block: right-hand sides per pass of
 * calls with nrhs > 1 (1 .. 32, default 16); groups: 0 = as many direction
 * groups as the device memory needs, >= 1 = about that many, and the grouped
 * layout also for single right-hand sides (for tests and memory limits). */
int defmm_set_blocking(defmm_handle* h, int rhs_block, int groups);
/* No counterpart in the reference.  on = 1: the mixed-precision path runs
 * the leaf interpolation GEMMs on the tensor cores (tcgen05 MMAs, 3-pass
 * split TF32, FP32 accumulation in tensor memory): P2M, M = Z W
 * (P2M.hpp:114-136), and L2P, p = Z^T X (L2P.hpp:122-173; target leaves of
 * at most 128 points) at orders <= 7; 0, and order 8 (where the equispaced
 * bases cancel too strongly for split TF32 to stay within 1e-6 of FP64):
 * CUDA-core FP32 FMAs.  The FP64 path always uses FP64 FMAs. */
int defmm_set_tensor_cores(defmm_handle* h, int on);
/* No counterpart in the reference.  Right-hand sides per M2L CTA of the
 * grouped layout (1, 2, 4, 8, default 4; capped by the order's register
 * budget and a divisor of the pass's right-hand sides): each
 * transfer-spectrum entry is read once for them.  Results are bit-identical
 * for every choice. */
int defmm_set_rhs_per_cta(defmm_handle* h, int rb);
/* No counterpart in the reference.  1: the grouped layout's mixed-precision
 * M2L at orders 3-6 stages spectra through shared memory with bulk copies
 * (cp.async.bulk), four consecutive target slots per CTA loading each
 * source's spectra once for all of them (M2L.hpp:115-127 with the targets'
 * lists merged); 0 (default, faster on the tested workloads): one target
 * slot per CTA, rhs_per_cta right-hand sides.  Results are bit-identical
 * either way. */
int defmm_set_m2l_staging(defmm_handle* h, int on);
/* No counterpart in the reference.  Wall time of each step of the last
 * prcmpt (octrees, levels and tables, the level walk's parts, slot lists,
 * near-field lists, transfer spectra) as text lines "seconds<TAB>step".
 * On entry *len is the capacity of buf (buf may be NULL); on return *len is
 * the size needed including the terminating zero. */
int defmm_setup_times(const defmm_handle* h, char* buf, int64_t* len);

/* No counterpart in the reference.  Independent operators (handles of
 * problems of any sizes, orders and wavenumbers) applied together: each
 * handle's matvec is captured as a CUDA graph (one run on its own stream, on
 * d_in[i] -> d_out[i], device pointers as in defmm_gemv_device) and becomes a
 * node of one graph, so one launch runs all of them.  The members are spread
 * over `lanes` >= 1 chains (largest first, onto the chain with the fewest
 * points so far): matvecs of one chain run in turn, chains run concurrently.
 * The handles and buffers must outlive the batch; after prcmpt,
 * defmm_set_precision, defmm_autotune, defmm_set_launch or
 * defmm_set_m2l_pairing on a member, create the batch again (it holds a copy of the member's graph).  Returns NULL on
 * failure (see the members' defmm_last_error). */
typedef struct defmm_batch defmm_batch;
defmm_batch* defmm_batch_create(int64_t n, defmm_handle* const* hs,
                                const void* const* d_in, void* const* d_out,
                                int lanes);
/* One launch of every member's matvec on `stream` (a cudaStream_t; NULL is
 * the legacy default stream), without synchronising. */
int defmm_batch_launch(defmm_batch* b, void* stream);
void defmm_batch_destroy(defmm_batch* b);

/* Many right-hand sides at once (host vectors, rhs-major), in passes as in
 * defmm_gemv_device. */
int defmm_gemv_batched(defmm_handle* h, int64_t nrhs, const double* in,
                       double* out);

/* friend CheckFULL(IBFMM_Mat&) (interface.hpp:178-221), sampled: FP64 direct
 * sum on the GPU at `nsamples` seeded random targets against the last gemv;
 * err = {rel. Linf, rel. L1, rel. L2} over the samples (the reference prints
 * the same three norms over all targets). */
int defmm_check_full(defmm_handle* h, int64_t nsamples, uint64_t seed,
                     double err[3]);

/* No counterpart in the reference.  FP64 direct sums, the arithmetic of
 * defmm_check_full, that allocate no device memory: out[t] = sum_j q_j
 * exp(i kappa |x_t - y_j|) / (4 pi |x_t - y_j|) over the handle's sources
 * y_j with the charges q_j of the last host gemv (its last right-hand side);
 * pairs with |x_t - y_j|^2 < 1e-16 (|x_t - y_j| < 1e-8) contribute zero, as in
 * the reference's CheckFULL.  d_targets: nt x 3 doubles, d_out: nt complex
 * doubles, both device pointers the caller owns; runs on `stream` (NULL = the
 * handle's own stream) without synchronising.
 *   - Scratch is a fixed 4 MiB array in the library's device image, so
 *     nt <= 262144 (DEFMM_ERR_ARG beyond, with a message).
 *   - The first call on a device looks up that array's address (a runtime
 *     query, no allocation); make one call before any stream capture that
 *     should contain it.  Outside a capture every call looks it up again.
 *   - All calls on one device share the scratch: calls that can overlap on
 *     the GPU (different streams, threads or handles) race and must be
 *     serialised by the caller.
 *   - The call reads the handle's device copy of the charges on `stream`;
 *     the handle's next host gemv waits for that read before overwriting
 *     them.  The calling thread's current device is left as it was. */
int defmm_direct_noalloc(defmm_handle* h, const double* d_targets, int64_t nt,
                         double* d_out, void* stream);

/* No counterpart in the reference.  Measurement helper: L2-to-SM read
 * bandwidth of the current device in GB/s (every SM streaming a buffer of
 * `bytes`, 1..96 MiB, that stays in L2, `reps` times; allocates and frees
 * the buffer).  The roofline denominator of the L2-bound M2L kernels. */
int defmm_probe_l2_read(int64_t bytes, int reps, double* gbs);

/* Sizes and statistics.  what: see DEFMM_INFO_* below. */
#define DEFMM_INFO_N_SOURCES 0
#define DEFMM_INFO_N_TARGETS 1
#define DEFMM_INFO_NLVL 2
#define DEFMM_INFO_CPT 3
#define DEFMM_INFO_MAX_STAGE 4
#define DEFMM_INFO_CELLS_T 5
#define DEFMM_INFO_CELLS_S 6
#define DEFMM_INFO_SLOTS_S 7
#define DEFMM_INFO_SLOTS_T 8
#define DEFMM_INFO_FAR_HF 9
#define DEFMM_INFO_FAR_LF 10
#define DEFMM_INFO_NEAR 11
#define DEFMM_INFO_I_NEAR 12
#define DEFMM_INFO_TABLES 13
#define DEFMM_INFO_DEVICE_BYTES 14
#define DEFMM_INFO_LIST_RECORDS 15 /* 1 if lists were recorded (parity) */
#define DEFMM_INFO_LAUNCHES 16     /* kernels launched by the last gemv call */
#define DEFMM_INFO_M2L_TARGETS 17  /* target slots receiving M2L */
#define DEFMM_INFO_LEAF_SLOTS_S 18 /* source leaf expansions (P2M outputs) */
#define DEFMM_INFO_PERMUTED_SPECTRA 19 /* (spectrum, symmetry) pairs used by M2L */
#define DEFMM_INFO_PLAN_WALK_DEVICE 20 /* 1 if prcmpt's level walk ran on the GPU */
#define DEFMM_INFO_PLAN_MS 21          /* prcmpt time (tree, lists, spectra), ms */
#define DEFMM_INFO_PLAN_WALK_MS 22     /* of which the level walk, ms */
#define DEFMM_INFO_M2L_THREADS 23      /* M2L threads per target slot (current precision) */
#define DEFMM_INFO_P2P_BLOCKS_PER_SM 24 /* near-field CTAs per SM (current precision) */
#define DEFMM_INFO_M2L_PAIRING 25       /* 1: two target slots per M2L CTA (current precision) */
#define DEFMM_INFO_LAYOUT 26            /* 0 none yet, 1 resident, 2 grouped */
#define DEFMM_INFO_RHS_BLOCK 27         /* right-hand sides per pass of the grouped layout */
#define DEFMM_INFO_GROUPS 28            /* direction groups of the grouped layout */
#define DEFMM_INFO_M2M_ENTRIES 29       /* (parent slot, child slot) transfers of M2M */
#define DEFMM_INFO_L2L_ENTRIES 30       /* (child slot, parent slot) transfers of L2L */
#define DEFMM_INFO_P2M_POINT_SLOTS 31   /* sum over source leaves of particles x slots */
#define DEFMM_INFO_L2P_POINT_SLOTS 32   /* sum over target leaves of particles x slots */
#define DEFMM_INFO_M2F_SLOTS 33         /* source slots transformed by M2F */
#define DEFMM_INFO_TENSOR_CORES 34      /* 1: mixed-precision P2M and L2P run on the tensor cores */
#define DEFMM_INFO_TREE_DEVICE 35       /* 1 if prcmpt ordered the octrees' particles on the GPU */
#define DEFMM_INFO_TREE_MS 36           /* prcmpt's octree build, ms */
#define DEFMM_INFO_RHS_PER_CTA 37       /* right-hand sides per M2L CTA of the grouped layout */
#define DEFMM_INFO_M2L_STAGING 38       /* 1: shared-memory-staged M2L with target groups enabled */
#define DEFMM_INFO_M2L_GROUP_LIST 39    /* longest list total of four consecutive target slots */
int defmm_info(const defmm_handle* h, int what, int64_t* value);

/* Per-phase device times (ms) of the last gemv, in this order:
 * P2M, M2M, M2F, M2L, F2L, L2L, L2P, P2P, gather+scatter, total.
 * F2L is fused into the M2L kernel and reads 0. */
int defmm_phase_times(const defmm_handle* h, double ms[10]);

/* Replay repeated matvecs from a captured CUDA graph (default on): the
 * first gemv with a given precision, input, output and stream captures the
 * launch sequence, later ones replay it.  on = 0 / 1. */
int defmm_set_graphs(defmm_handle* h, int on);

/* Per-phase timing with CUDA events (adds synchronisation between phases;
 * off by default).  on = 0 / 1. */
int defmm_set_profiling(defmm_handle* h, int on);

/* Record the interaction lists at the next prcmpt (costs host memory; for
 * parity checks against the reference). */
int defmm_keep_lists(defmm_handle* h, int on);

/* No counterpart in the reference (its precomputation is host-only).  on != 0
 * (the default): prcmpt runs the level walk of the plan — dual traversal,
 * cones, effective directions, slots, far-field entries — and the lists built
 * from it (transfer, per-cell slot and near-field lists) on the GPU when one
 * is present, with results identical to the host build; on == 0: always on
 * the host.  List records (defmm_keep_lists) always come from the host walk. */
int defmm_set_plan_device(defmm_handle* h, int on);

/* No counterpart in the reference.  Autotuner: on this operator and its
 * current precision, `reps` times three timing runs on the handle's own
 * buffers, one per near-field candidate (8, 16 or 32 CTAs per SM, timed on
 * the near-field phase); the first also runs the M2L of every level holding
 * at least 2% of the far pairs in 16 interleaved slices of its target slots,
 * slice i with candidate i mod 4 (128 or 256 threads per CTA, one or two
 * target slots per CTA), and each level keeps the candidate with the least
 * time per far pair (the other levels take the busiest level's).  Every
 * choice gives bit-identical results.  The choice of the level with the
 * most far pairs and the near-field CTAs per SM are written to choice[2]
 * when not NULL (also DEFMM_INFO_M2L_THREADS / DEFMM_INFO_M2L_PAIRING /
 * DEFMM_INFO_P2P_BLOCKS_PER_SM; every level's: defmm_m2l_schedule); the next
 * matvec captures a new graph.  Choices are cached per operator shape in the
 * process. */
int defmm_autotune(defmm_handle* h, int reps, int32_t* choice);
/* No counterpart in the reference.  The M2L launch choice of levels
 * 0 .. n-1 for the current precision: threads[l] per CTA and pairing[l]
 * (1: two target slots per CTA). */
int defmm_m2l_schedule(const defmm_handle* h, int32_t* threads, int32_t* pairing, int n);
/* No counterpart in the reference.  Sets the same launch choices by hand for
 * the current precision: m2l_threads 128 or 256 (0: the order's default),
 * p2p_blocks_per_sm 1..64 (0: 16). */
int defmm_set_launch(defmm_handle* h, int m2l_threads, int p2p_blocks_per_sm);
/* No counterpart in the reference.  on = 1: each M2L CTA takes two
 * consecutive target slots and reads a source spectrum the two share once
 * (current precision); 0: one slot per CTA. */
int defmm_set_m2l_pairing(defmm_handle* h, int on);

/* Tree dump in the layout of the reference's cell array (SourceRoot /
 * TargetRoot, interface.hpp:174-175; cells in depth-first pre-order):
 * which = 0 targets, 1 sources.  cells_int: 8 int32 per cell (idx0, idx1,
 * idx2, lvl, nprt, first particle, number of sons, number of expansions);
 * cells_dbl: 4 doubles per cell (ctr0, ctr1, ctr2, rad); dirs: effective
 * directions of every cell, concatenated in cell order (may be NULL to query
 * the count, returned in *ndirs); perm: user index of each tree-order
 * particle.  Any output pointer may be NULL. */
int defmm_dump_tree(const defmm_handle* h, int which, int32_t* cells_int,
                    double* cells_dbl, int32_t* dirs, int64_t* ndirs,
                    int32_t* perm);

/* Recorded lists (defmm_keep_lists): far HF records (t, s, lvl, cone, iz,
 * hash), far LF records (t, s, lvl, iz, hash), near records (t, s); counts
 * in n[3].  Pointers may be NULL to query the counts. */
int defmm_dump_lists(const defmm_handle* h, int32_t* far_hf, int32_t* far_lf,
                     int32_t* near_, int64_t n[3]);

/* No counterpart in the reference (its M2L tables are per-cell pointers,
 * M2L.hpp:41-83).  The far-field work as the matvec runs it: per target
 * slot (CSR ptr, n[0] = target slots + 1 entries) the source slots and the
 * transfer spectra as (table index << 6) | symmetry hash, n[1] entries each,
 * sorted by source slot within a target slot.  Identical whether prcmpt's
 * level walk ran on the GPU or on the host.  Pointers may be NULL to query
 * the counts. */
int defmm_dump_m2l(const defmm_handle* h, int64_t* ptr, int32_t* src,
                   uint32_t* tab, int64_t n[2]);

/* No counterpart in the reference (its near field walks the P2P lists of
 * each target leaf, P2P.hpp:43-79).  Fingerprints of the near-field work
 * lists as the matvec runs them, for parity checks of the device plan
 * against the host plan: digest[0..22] are 64-bit FNV-1a hashes of the
 * chunk, work-item, symmetric-block and reduction arrays (count and bytes),
 * digest[23..25] the scratch size, the particle interactions and the near
 * pairs.  Identical whether prcmpt built the lists on the GPU or on the
 * host. */
int defmm_near_digest(const defmm_handle* h, uint64_t digest[26]);

/* No counterpart in the reference.  Order-selection network (learned.py):
 * a perceptron DEFMM_MLP_IN -> DEFMM_MLP_HIDDEN -> DEFMM_MLP_HIDDEN ->
 * DEFMM_MLP_OUT (ReLU, ReLU, logits over interpolation orders 3..8) that
 * predicts the lowest order meeting a requested accuracy from problem
 * features.  Parameters: one flat FP32 array of DEFMM_MLP_PARAMS values,
 * W1 (64 x 12, row-major), b1, W2 (64 x 64), b2, W3 (6 x 64), b3.  All
 * pointers are device pointers; calls run on `stream` (a cudaStream_t, NULL
 * the legacy default stream) without synchronising. */
#define DEFMM_MLP_IN 12
#define DEFMM_MLP_HIDDEN 64
#define DEFMM_MLP_OUT 6
#define DEFMM_MLP_PARAMS 5382
/* FP32 forward of n samples X (n x 12): activations H1, H2 (n x 64), logits
 * (n x 6). */
int defmm_mlp_forward(const float* params, const float* X, int64_t n, float* H1,
                      float* H2, float* logits, void* stream);
/* Gradient of the weighted softmax cross-entropy
 * sum_i w_i (-log softmax(logits_i)[y_i]) / wsum (w NULL: all 1) into grads
 * (DEFMM_MLP_PARAMS floats) and its value into *loss (device float);
 * scratch: n * (6 + 2 * 64) floats. */
int defmm_mlp_backward(const float* params, const float* X, const float* H1,
                       const float* H2, const float* logits, const int32_t* y,
                       const float* w, float wsum, int64_t n, float* grads,
                       float* loss, float* scratch, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected at `step` >= 1)
 * on params with moments m, v, and decoupled weight decay wd >= 0:
 * p -= lr (mhat / (sqrt(vhat) + eps) + wd p). */
int defmm_mlp_adam(float* params, const float* grads, float* m, float* v,
                   int64_t step, float lr, float wd, void* stream);
/* BF16 copy of the parameters (round to nearest even), for inference. */
int defmm_mlp_to_bf16(const float* params, uint16_t* out, void* stream);
/* Inference with BF16 parameters and FP32 accumulation: logits (n x 6). */
int defmm_mlp_infer_bf16(const uint16_t* params_bf16, const float* X, int64_t n,
                         float* logits, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DEFMM_B200_H */
