// Operator handle: host plan -> device arrays, matvec orchestration, C ABI.
#include <algorithm>
#include <array>
#include <chrono>
#include <climits>
#include <map>
#include <memory>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/defmm_b200.h"
#include "engine_internal.h"
#include "fmm_kernels.h"
#include "plan.hpp"
#include "plan_device.hpp"

using dfb::DevPlan;
using dfb::Plan;
using dfb::Levels;

namespace {

enum Phase { PH_P2M = 0, PH_M2M, PH_M2F, PH_M2L, PH_F2L, PH_L2L, PH_L2P, PH_P2P, PH_SCATTER, PH_TOTAL, PH_N };

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

// Direction-streamed layout with right-hand-side blocks (no counterpart in
// the reference, whose expansions are all resident).  The HF levels' slots
// are split into groups by direction at the deepest HF level (the pivot):
// direction c there owns directions [c f, (c + 1) f) at a level with f times
// more directions, and M2M, M2L and L2L never leave a group.  One group's M
// and L (R right-hand sides per slot) are on the device at a time; LF levels
// (below the pivot, one slot per cell) stay resident.
struct GroupedLayout {
  int R = 0;                        // right-hand sides per slot
  std::vector<int> hl;              // HF levels holding slots, coarse to fine
  int lh = -1;                      // pivot (deepest HF level), -1: none
  std::vector<int64_t> fl;          // per level of hl: directions per pivot direction
  std::vector<std::pair<int, int>> groups;  // pivot direction ranges [c0, c1)
  int64_t gS_max = 0, gT_max = 0;   // slots of the largest group (S, T)
  int64_t lfS0 = 0, lfS1 = 0, lfT0 = 0, lfT1 = 0;  // LF slot ranges
  int64_t f_cap = 0;                // source slots per F batch
  DevBuf Mg, Lg, Mlf, Llf, F, q, pnear, pfar, tpart;
};

struct defmm_handle {
  std::vector<double> src, trg;  // user-order coordinates
  Plan plan;
  bool built = false;
  bool uploaded = false;
  bool keep_lists = false;
  bool plan_device = true;   // run the plan's level walk on the GPU when one is present
  bool walked_on_device = false;
  int precision = DEFMM_PRECISION_FP64;
  std::string err;
  // device state
  int device = -1;
  cudaStream_t st = nullptr, st2 = nullptr;  // own stream; near field
  cudaStream_t cur = nullptr;                // stream of the gemv in progress (phase events)
  std::vector<void*> plan_allocs;  // freed when the plan is rebuilt
  DevPlan dp;
  const dfb::OpTable* ops = nullptr;
  int ops_prec = -1;
  // precision-dependent arrays
  DevBuf M, Lx, F, q, sig, sig2, ptab;
  const uint32_t* d_ptab_key = nullptr;
  int64_t f_cap = 0;  // source slots per F batch buffer
  // FP64 vectors
  DevBuf pnear, pfar, qin, out, chk;
  DevBuf rin, rout;  // staging of device multi-RHS calls (defmm_gemv_device, nrhs > 1)
  const int32_t *d_p2m_leaf = nullptr, *d_l2p_leaf = nullptr;
  const int32_t *d_tfirst = nullptr, *d_tn = nullptr, *d_sfirst = nullptr, *d_sn = nullptr;
  const int64_t* d_p2p_ptr = nullptr;
  const int32_t* d_p2p_order = nullptr;
  const int32_t *d_p2p_item_chunk = nullptr, *d_sym_item_chunk = nullptr;
  const int64_t *d_p2p_chunk_items = nullptr, *d_sym_chunk_items = nullptr;
  double2* d_tpart = nullptr;  // near-field item partial sums (32 per item)
  unsigned long long* d_queue = nullptr;
  // symmetric near field (Plan::self_*, sym_*, red_*)
  const int64_t *d_self_ptr = nullptr, *d_sym_ptr = nullptr, *d_sym_soff = nullptr, *d_red_ptr = nullptr,
                *d_red_off = nullptr;
  const int32_t *d_self_sfirst = nullptr, *d_self_sn = nullptr, *d_self_order = nullptr;
  const int32_t *d_sym_sfirst = nullptr, *d_sym_sn = nullptr, *d_sym_order = nullptr;
  const int32_t *d_red_first = nullptr, *d_red_n = nullptr;
  DevBuf pscr;           // source-side partial sums (one complex per slot)
  bool use_sym = false;  // this precision runs the symmetric near field
  int nsm = 148;
  // launch choices (defmm_autotune), per precision: M2L threads per target
  // slot (0: the order's default) and near-field CTAs per SM
  int m2l_nt[2] = {0, 0};
  int m2l_pair[2] = {0, 0};  // two target slots per M2L CTA
  // per-level choices of the autotuner (per precision; < 0: the values above)
  int16_t m2l_lvl_nt[2][32], m2l_lvl_pair[2][32];

  int p2p_bps[2] = {16, 16};
  int64_t nchunk = 0;
  size_t dev_bytes = 0;
  // layout of the expansions: 0 none, 1 resident (every slot's M and L),
  // 2 grouped (GroupedLayout)
  int layout = 0;
  GroupedLayout gl;
  int rhs_block = 16;     // right-hand sides per pass of multi-RHS calls
  int rhs_block_m2l = 4;  // right-hand sides per M2L CTA (capped by the order)
  bool m2l_staging = false;  // grouped layout, FP32: shared-memory-staged M2L with target groups
  int tune_level = -1;        // >= 0: timing runs of the autotuner (see run_gemv)
  int tune_m2l = 0;           // 1: the timing run also times the M2L candidates
  bool tune_lvl_on[32];       // levels whose M2L the timing runs execute
  double tune_ms[32][4], tune_pairs[32][4];  // per (level, M2L candidate): time, far pairs
  int64_t m2l_lgroup = 0;   // longest list total of kM2LGroup consecutive target slots
  bool use_tc = false;    // mixed precision: P2M on the tensor cores (tcgen05)
  int groups_forced = 0;  // > 0: direction groups requested (also for one RHS)
  int groups_used = 0;    // groups of the last grouped pass
  // leaves at precomputed levels sorted by level (P2M: sources, L2P: targets)
  const int32_t *d_p2m_bylvl = nullptr, *d_l2p_bylvl = nullptr;
  std::vector<int64_t> p2m_lvl_off, l2p_lvl_off;  // nlvl + 1 offsets
  int l2p_max_points = 0;  // largest target leaf at a precomputed level
  double phase_ms[PH_N] = {0};
  cudaEvent_t ev[2 * PH_N] = {};
  cudaEvent_t ev_ready = nullptr, ev_done = nullptr;  // cross-stream ordering
  // recorded by defmm_direct_noalloc after its last read of qin (on the
  // caller's stream); the next host gemv waits for it before overwriting qin
  cudaEvent_t ev_qin_read = nullptr;
  bool events = false;
  bool has_out = false;
  int64_t launches = 0;  // kernels launched by the last gemv call
  // CUDA graph of one matvec, replayed while (precision, input, output,
  // stream) stay the same
  bool use_graphs = true;
  cudaGraph_t graph = nullptr;  // the captured matvec behind gexec (child node of batches)
  cudaGraphExec_t gexec = nullptr;
  const void* g_in = nullptr;
  void* g_out = nullptr;
  cudaStream_t g_stream = nullptr;
  int g_prec = -1;
  int64_t g_launches = 0;

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
};

namespace {

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      return h->fail(e_ == cudaErrorMemoryAllocation ? DEFMM_ERR_MEMORY : DEFMM_ERR_CUDA,     \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                   \
    }                                                                                        \
  } while (0)

void free_buf(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

// The autotuner's M2L candidates: (two target slots per CTA, threads per CTA)
constexpr int kM2LCand[4][2] = {{0, 128}, {0, 256}, {1, 128}, {1, 256}};

// M2L launch choice of level l (the autotuner's per-level pick, else the
// operator-wide one)
void m2l_choice(const defmm_handle* h, int pi, int l, int* nt, int* pair) {
  *nt = h->m2l_lvl_nt[pi][l] >= 0 ? h->m2l_lvl_nt[pi][l] : h->m2l_nt[pi];
  *pair = h->m2l_lvl_pair[pi][l] >= 0 ? h->m2l_lvl_pair[pi][l] : h->m2l_pair[pi];
}
void m2l_levels_reset(defmm_handle* h, int pi) {
  for (int l = 0; l < 32; l++) h->m2l_lvl_nt[pi][l] = h->m2l_lvl_pair[pi][l] = -1;
}

int ensure(defmm_handle* h, DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes && b.p) return 0;
  free_buf(b);
  if (!bytes) return 0;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    b.p = nullptr;
    cudaGetLastError();
    return h->fail(DEFMM_ERR_MEMORY, "cudaMalloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
  }
  b.bytes = bytes;
  return 0;
}

template <typename V>
int upload(defmm_handle* h, const std::vector<V>& v, const V** out) {
  *out = nullptr;
  if (v.empty()) return 0;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, v.size() * sizeof(V));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return h->fail(DEFMM_ERR_MEMORY, std::string("device allocation failed: ") + cudaGetErrorString(e));
  }
  h->plan_allocs.push_back(p);
  h->dev_bytes += v.size() * sizeof(V);
  e = cudaMemcpy(p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return h->fail(DEFMM_ERR_CUDA, cudaGetErrorString(e));
  *out = static_cast<const V*>(p);
  return 0;
}

template <typename V>
std::vector<int32_t> to_i32(const std::vector<V>& v) {
  return std::vector<int32_t>(v.begin(), v.end());
}

void drop_graph(defmm_handle* h) {
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->gexec = nullptr;
  h->graph = nullptr;
  h->g_prec = -1;
}

void free_grouped(defmm_handle* h) {
  GroupedLayout& g = h->gl;
  for (DevBuf* b : {&g.Mg, &g.Lg, &g.Mlf, &g.Llf, &g.F, &g.q, &g.pnear, &g.pfar, &g.tpart}) free_buf(*b);
  g = GroupedLayout();
}

void free_plan_device(defmm_handle* h) {
  drop_graph(h);
  for (void* p : h->plan_allocs) cudaFree(p);
  h->plan_allocs.clear();
  free_buf(h->M);
  free_buf(h->Lx);
  free_buf(h->F);
  free_buf(h->q);
  free_buf(h->sig);
  free_buf(h->sig2);
  free_buf(h->ptab);
  free_buf(h->pnear);
  free_buf(h->pfar);
  free_buf(h->qin);
  free_buf(h->out);
  free_buf(h->rin);
  free_buf(h->rout);
  free_buf(h->chk);
  free_buf(h->pscr);
  free_grouped(h);
  h->layout = 0;
  h->use_sym = false;
  h->ops_prec = -1;
  h->dev_bytes = 0;
  h->has_out = false;
}

int upload_plan(defmm_handle* h) {
  Plan& p = h->plan;
  DevPlan& d = h->dp;
  std::memset(&d, 0, sizeof(d));
  int st;
#define UP(vec, field)                         \
  do {                                         \
    if ((st = upload(h, (vec), &(field)))) return st; \
  } while (0)
  std::vector<double4> c4(p.S.ncell);
  for (int64_t c = 0; c < p.S.ncell; c++)
    c4[c] = make_double4(p.S.ctr[3 * c], p.S.ctr[3 * c + 1], p.S.ctr[3 * c + 2], p.S.rad[c]);
  UP(c4, d.S_ctr);
  c4.resize(p.T.ncell);
  for (int64_t c = 0; c < p.T.ncell; c++)
    c4[c] = make_double4(p.T.ctr[3 * c], p.T.ctr[3 * c + 1], p.T.ctr[3 * c + 2], p.T.rad[c]);
  UP(c4, d.T_ctr);
  std::vector<double4>().swap(c4);
  UP(p.S.first, d.S_first);
  UP(p.S.nprt, d.S_nprt);
  UP(p.S.lvl, d.S_lvl);
  UP(p.T.first, d.T_first);
  UP(p.T.nprt, d.T_nprt);
  UP(p.T.lvl, d.T_lvl);
  UP(p.T.parent, d.T_parent);
  UP(p.S.pos, d.S_pos);
  UP(p.T.pos, d.T_pos);
  UP(p.S.perm, d.S_perm);
  UP(p.T.perm, d.T_perm);
  if (p.dev_scell_S) {  // built on the device by prcmpt
    d.sS_cell = static_cast<const int32_t*>(p.dev_scell_S);
    d.sS_dir = static_cast<const int32_t*>(p.dev_sdir_S);
    d.sT_cell = static_cast<const int32_t*>(p.dev_scell_T);
    d.sT_dir = static_cast<const int32_t*>(p.dev_sdir_T);
    h->dev_bytes += (size_t)(p.sS.n + p.sT.n) * 8;
  } else {
    UP(p.sS.cell, d.sS_cell);
    UP(p.sS.dir, d.sS_dir);
    UP(p.sT.cell, d.sT_cell);
    UP(p.sT.dir, d.sT_dir);
  }
  UP(p.sS.cell_ptr, d.S_cptr);
  UP(p.sT.cell_ptr, d.T_cptr);
  if (p.dev_cslot_S) {  // built on the device by prcmpt
    d.S_cslot = static_cast<const int32_t*>(p.dev_cslot_S);
    d.S_cdir = static_cast<const int32_t*>(p.dev_cdir_S);
    d.T_cslot = static_cast<const int32_t*>(p.dev_cslot_T);
    d.T_cdir = static_cast<const int32_t*>(p.dev_cdir_T);
    h->dev_bytes += (size_t)(p.sS.n + p.sT.n) * 8;
  } else {
    UP(to_i32(p.sS.cell_slots), d.S_cslot);
    UP(p.sS.cell_dirs, d.S_cdir);
    UP(to_i32(p.sT.cell_slots), d.T_cslot);
    UP(p.sT.cell_dirs, d.T_cdir);
  }
  if (p.dev_m2m_ptr) {  // built on the device by prcmpt
    d.m2m_ptr = static_cast<const int64_t*>(p.dev_m2m_ptr);
    d.m2m_child = static_cast<const int32_t*>(p.dev_m2m_child);
    d.l2l_ptr = static_cast<const int64_t*>(p.dev_l2l_ptr);
    d.l2l_parent = static_cast<const int32_t*>(p.dev_l2l_parent);
    h->dev_bytes += (size_t)(p.sS.n + p.sT.n + 2) * 8 + (size_t)(p.n_m2m + p.n_l2l) * 4;
  } else {
    UP(p.m2m_ptr, d.m2m_ptr);
    UP(p.m2m_child, d.m2m_child);
    UP(p.l2l_ptr, d.l2l_ptr);
    UP(p.l2l_parent, d.l2l_parent);
  }
  UP(p.m2l_ptr, d.m2l_ptr);
  if (p.dev_m2l_src) {  // built on the device by prcmpt
    d.m2l_src = static_cast<const int32_t*>(p.dev_m2l_src);
    d.m2l_tab = static_cast<const uint32_t*>(p.dev_m2l_tab);
    h->dev_bytes += (size_t)p.n_m2l * 8;
  } else {
    UP(p.m2l_src, d.m2l_src);
    UP(p.m2l_tab, d.m2l_tab);
  }
  UP(p.perm, d.perm);
  UP(p.ptab_key, h->d_ptab_key);
  std::vector<double> dirs;
  for (size_t e = 0; e < p.dirs.size() && e < 32; e++) {
    d.dir_off[e] = (int64_t)(dirs.size() / 3);
    dirs.insert(dirs.end(), p.dirs[e].begin(), p.dirs[e].end());
  }
  if (dirs.empty()) dirs.assign(3, 0.);
  UP(dirs, d.dirs);
  int64_t off = 0;
  for (size_t e = 0; e < p.sig.size() && e < 32; e++) {
    d.sig_off[e] = off;
    off += (int64_t)p.sig[e].size();
  }
  for (int l = 0; l < p.lv.nlvl && l < 32; l++) {
    d.ishf[l] = (int8_t)(p.lv.isHF[l] ? 1 : 0);
    d.hfstage[l] = (int8_t)p.lv.HFStage[l];
  }
  d.kappa = p.kappa;
  d.nlvl = p.lv.nlvl;
  UP(p.p2m_leaf, h->d_p2m_leaf);
  UP(p.l2p_leaf, h->d_l2p_leaf);
  {  // the same leaves grouped by level (stable), for per-level launches
    auto bylvl = [&](const std::vector<int32_t>& lv, const std::vector<int32_t>& leaves, std::vector<int32_t>& out,
                     std::vector<int64_t>& off) {
      off.assign(p.lv.nlvl + 1, 0);
      for (int32_t c : leaves) off[lv[c] + 1]++;
      for (int l = 0; l < p.lv.nlvl; l++) off[l + 1] += off[l];
      out.assign(leaves.size(), 0);
      std::vector<int64_t> pos(off.begin(), off.end() - 1);
      for (int32_t c : leaves) out[pos[lv[c]]++] = c;
    };
    h->l2p_max_points = 0;
    for (int32_t c : p.l2p_leaf) h->l2p_max_points = std::max(h->l2p_max_points, (int)p.T.nprt[c]);
    std::vector<int32_t> tmp;
    bylvl(p.S.lvl, p.p2m_leaf, tmp, h->p2m_lvl_off);
    UP(tmp, h->d_p2m_bylvl);
    bylvl(p.T.lvl, p.l2p_leaf, tmp, h->l2p_lvl_off);
    UP(tmp, h->d_l2p_bylvl);
  }
  if (p.nd.on) {  // built on the device by prcmpt
    const Plan::NearOnDevice& n = p.nd;
    h->d_tfirst = n.tfirst;
    h->d_tn = n.tn;
    h->d_p2p_ptr = n.p2p_ptr;
    h->d_sfirst = n.p2p_sfirst;
    h->d_sn = n.p2p_sn;
    h->d_p2p_order = n.p2p_order;
    h->d_p2p_item_chunk = n.p2p_item_chunk;
    h->d_p2p_chunk_items = n.p2p_chunk_items;
    if (p.p2p_sym) {
      h->d_sym_item_chunk = n.sym_item_chunk;
      h->d_sym_chunk_items = n.sym_chunk_items;
      h->d_self_ptr = n.self_ptr;
      h->d_self_sfirst = n.self_sfirst;
      h->d_self_sn = n.self_sn;
      h->d_self_order = n.self_order;
      h->d_sym_ptr = n.sym_ptr;
      h->d_sym_sfirst = n.sym_sfirst;
      h->d_sym_sn = n.sym_sn;
      h->d_sym_soff = n.sym_soff;
      h->d_sym_order = n.sym_order;
      h->d_red_first = n.red_first;
      h->d_red_n = n.red_n;
      h->d_red_ptr = n.red_ptr;
      h->d_red_off = n.red_off;
    }
  } else {
    UP(p.p2p_tfirst, h->d_tfirst);
    UP(p.p2p_tn, h->d_tn);
    UP(p.p2p_ptr, h->d_p2p_ptr);
    UP(p.p2p_sfirst, h->d_sfirst);
    UP(p.p2p_sn, h->d_sn);
    UP(p.p2p_order, h->d_p2p_order);
    UP(p.p2p_item_chunk, h->d_p2p_item_chunk);
    UP(p.p2p_chunk_items, h->d_p2p_chunk_items);
    if (p.p2p_sym) {
      UP(p.sym_item_chunk, h->d_sym_item_chunk);
      UP(p.sym_chunk_items, h->d_sym_chunk_items);
      UP(p.self_ptr, h->d_self_ptr);
      UP(p.self_sfirst, h->d_self_sfirst);
      UP(p.self_sn, h->d_self_sn);
      UP(p.self_order, h->d_self_order);
      UP(p.sym_ptr, h->d_sym_ptr);
      UP(p.sym_sfirst, h->d_sym_sfirst);
      UP(p.sym_sn, h->d_sym_sn);
      UP(p.sym_soff, h->d_sym_soff);
      UP(p.sym_order, h->d_sym_order);
      UP(p.red_first, h->d_red_first);
      UP(p.red_n, h->d_red_n);
      UP(p.red_ptr, h->d_red_ptr);
      UP(p.red_off, h->d_red_off);
    }
  }
  h->nchunk = p.near_chunks();
#undef UP
  {
    void* e = nullptr;
    CK(cudaMalloc(&e, sizeof(int)));
    h->plan_allocs.push_back(e);
    CK(cudaMemset(e, 0, sizeof(int)));
    d.err = static_cast<int*>(e);
    const size_t nitem = (size_t)std::max<int64_t>(1, std::max(p.near_items(), p.near_sym_items()));
    void* tp = nullptr;
    CK(cudaMalloc(&tp, nitem * 32 * sizeof(double2)));
    h->plan_allocs.push_back(tp);
    h->dev_bytes += nitem * 32 * sizeof(double2);
    h->d_tpart = static_cast<double2*>(tp);
    void* qc = nullptr;
    CK(cudaMalloc(&qc, 2 * sizeof(unsigned long long)));  // P2P (stream 2), M2L (main stream)
    h->plan_allocs.push_back(qc);
    h->d_queue = static_cast<unsigned long long*>(qc);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, dev));
  }
  int64_t nS = (int64_t)p.S.perm.size(), nT = (int64_t)p.T.perm.size();
  if ((st = ensure(h, h->pnear, 16 * nT)) || (st = ensure(h, h->pfar, 16 * nT)) ||
      (st = ensure(h, h->qin, 16 * nS)) || (st = ensure(h, h->out, 16 * nT)))
    return st;
  return 0;
}

// Tables whose element type follows the precision: the order's kernels and
// constant tables, signatures, permuted transfer spectra.  Releases the
// expansion layout of the previous precision.
int prepare_tables(defmm_handle* h) {
  if (h->ops_prec == h->precision) return 0;
  drop_graph(h);
  Plan& p = h->plan;
  const bool fp64 = h->precision == DEFMM_PRECISION_FP64;
  const size_t cs = fp64 ? 16 : 8;
  free_buf(h->M);
  free_buf(h->Lx);
  free_buf(h->F);
  free_buf(h->q);
  free_buf(h->sig);
  free_buf(h->sig2);
  free_buf(h->ptab);
  free_buf(h->pscr);
  free_grouped(h);
  h->layout = 0;
  h->use_sym = false;
  h->ops = dfb::op_table(p.L, fp64);
  if (!h->ops) return h->fail(DEFMM_ERR_ARG, "unsupported order");
  std::vector<double> mats;
  for (int k = 0; k < 2; k++) mats.insert(mats.end(), p.m2m[k].begin(), p.m2m[k].end());
  for (int k = 0; k < 2; k++) mats.insert(mats.end(), p.l2l[k].begin(), p.l2l[k].end());
  CK(h->ops->setup(mats.data()));
  CK(dfb::setup_rhs_kernels());
  if (!fp64) CK(dfb::setup_tc_kernels());
  auto put = [&](DevBuf& b, const dfb::cplx* src, size_t n) -> int {
    int st = ensure(h, b, std::max<size_t>(1, n) * cs);
    if (st) return st;
    if (!n) return 0;
    if (fp64) {
      CK(cudaMemcpy(b.p, src, n * 16, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(2 * n);
      for (size_t i = 0; i < n; i++) {
        f[2 * i] = (float)src[i].real();
        f[2 * i + 1] = (float)src[i].imag();
      }
      CK(cudaMemcpy(b.p, f.data(), n * 8, cudaMemcpyHostToDevice));
    }
    return 0;
  };
  int st;
  DevBuf base;  // transfer spectra, tables x PP, in the precision's complex type
  if (p.tables_on_device) {
    // spectra and signatures computed on the device in FP64 (bit-identical
    // to the host's), then rounded to FP32 for the mixed path
    size_t nsig = 0;
    for (size_t e = 0; e < p.sig.size() && e < 32; e++) nsig += p.sig[e].size();
    const size_t ntabv = p.tab_fund.size() * (size_t)p.PP;
    DevBuf t64, a64, b64;
    if ((st = ensure(h, t64, std::max<size_t>(1, ntabv) * 16)) || (st = ensure(h, a64, std::max<size_t>(1, nsig) * 16)) ||
        (st = ensure(h, b64, std::max<size_t>(1, nsig) * 16))) {
      free_buf(t64);
      free_buf(a64);
      free_buf(b64);
      return st;
    }
    std::string e;
    st = dfb::device_plan_tables(p, (double2*)t64.p, (double2*)a64.p, (double2*)b64.p, e);
    if (st) {
      free_buf(t64);
      free_buf(a64);
      free_buf(b64);
      return h->fail(DEFMM_ERR_CUDA, e);
    }
    if (fp64) {
      std::swap(h->sig, a64);
      std::swap(h->sig2, b64);
      std::swap(base, t64);
    } else {
      if ((st = ensure(h, h->sig, std::max<size_t>(1, nsig) * 8)) ||
          (st = ensure(h, h->sig2, std::max<size_t>(1, nsig) * 8)) || (st = ensure(h, base, std::max<size_t>(1, ntabv) * 8))) {
        free_buf(t64);
        free_buf(a64);
        free_buf(b64);
        return st;
      }
      dfb::tables_to_float((const double2*)a64.p, (float2*)h->sig.p, (int64_t)nsig, h->st);
      dfb::tables_to_float((const double2*)b64.p, (float2*)h->sig2.p, (int64_t)nsig, h->st);
      dfb::tables_to_float((const double2*)t64.p, (float2*)base.p, (int64_t)ntabv, h->st);
      CK(cudaStreamSynchronize(h->st));
    }
    free_buf(t64);
    free_buf(a64);
    free_buf(b64);
  } else {
    std::vector<dfb::cplx> s1, s2;
    for (size_t e = 0; e < p.sig.size() && e < 32; e++) {
      s1.insert(s1.end(), p.sig[e].begin(), p.sig[e].end());
      s2.insert(s2.end(), p.sig2[e].begin(), p.sig2[e].end());
    }
    if ((st = put(h->sig, s1.data(), s1.size())) || (st = put(h->sig2, s2.data(), s2.size())) ||
        (st = put(base, p.tables.data(), p.tables.size())))
      return st;
  }
  {
    // permuted spectra used by M2L, gathered once on the device
    const int64_t np = (int64_t)p.ptab_key.size();
    if ((st = ensure(h, h->ptab, std::max<int64_t>(1, np) * p.PP * cs + 16))) {  // + slack as for F
      free_buf(base);
      return st;
    }
    h->ops->permute(np, h->d_ptab_key, h->dp.perm, base.p, h->ptab.p, h->st);
    CK(cudaStreamSynchronize(h->st));
    free_buf(base);
  }
  h->ops_prec = h->precision;
  return 0;
}

// Largest cone (source slots) of any precomputed level: the smallest F batch.
int64_t largest_cone(const Plan& p) {
  int64_t need = 1;
  for (int l = 0; l < p.lv.nlvl; l++) {
    const auto& cS = p.sS.cone_begin[l];
    for (size_t c = 0; c + 1 < cS.size(); c++) need = std::max(need, cS[c + 1] - cS[c]);
  }
  return need;
}

// Device bytes of the resident layout: every slot's M and L, charges, the
// smallest F batch.
size_t resident_bytes(const defmm_handle* h) {
  const Plan& p = h->plan;
  const size_t cs = h->precision == DEFMM_PRECISION_FP64 ? 16 : 8;
  return (size_t)(p.sS.n + p.sT.n) * p.LL * cs + p.S.perm.size() * cs + (size_t)largest_cone(p) * p.PP * cs;
}

// Resident layout: M and L of every slot.  Releases a grouped layout first.
int prepare_resident(defmm_handle* h) {
  if (h->layout == 1) return 0;
  drop_graph(h);
  free_grouped(h);
  h->layout = 0;
  Plan& p = h->plan;
  const bool fp64 = h->precision == DEFMM_PRECISION_FP64;
  const size_t cs = fp64 ? 16 : 8;
  int st;
  const int64_t nS = (int64_t)p.S.perm.size();
  if ((st = ensure(h, h->M, std::max<int64_t>(1, p.sS.n) * p.LL * cs)) ||
      (st = ensure(h, h->Lx, std::max<int64_t>(1, p.sT.n) * p.LL * cs)) || (st = ensure(h, h->q, nS * cs)))
    return st;
  // symmetric near field when its scratch takes at most 70% of the free
  // memory and can be allocated (otherwise every interaction is evaluated
  // from both sides)
  free_buf(h->pscr);
  h->use_sym = false;
  if (p.p2p_sym && p.sym_scratch > 0) {
    size_t fr0 = 0, tot0 = 0;
    CK(cudaMemGetInfo(&fr0, &tot0));
    const size_t b = (size_t)p.sym_scratch * cs;
    if (b <= (size_t)(0.7 * (double)fr0)) {
      void* ptr = nullptr;
      if (cudaMalloc(&ptr, b) == cudaSuccess) {
        h->pscr.p = ptr;
        h->pscr.bytes = b;
        h->use_sym = true;
      } else {
        cudaGetLastError();
      }
    }
  }
  // F batch buffer: at least the largest cone of any level, at most about
  // half of the free memory
  int64_t need = largest_cone(p), want = 0;
  for (int l = 0; l < p.lv.nlvl; l++) {
    const auto& cS = p.sS.cone_begin[l];
    want = std::max(want, cS.back() - cS.front());
  }
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  const size_t per = (size_t)p.PP * cs;
  int64_t cap = (int64_t)((fr * 0.5) / per);
  cap = std::min<int64_t>(cap, (int64_t)((size_t)64 << 30) / (int64_t)per);
  cap = std::min(cap, std::max(want, need));
  if (cap < need) return h->fail(DEFMM_ERR_MEMORY, "not enough device memory for one cone of spectra");
  h->f_cap = cap;
  if ((st = ensure(h, h->F, cap * per))) return st;
  h->layout = 1;
  return 0;
}

int prepare_precision(defmm_handle* h) {
  int st = prepare_tables(h);
  if (st) return st;
  return prepare_resident(h);
}

// Slot ranges of one direction group at HF level hl[i]: S [*s0, *s1),
// T [*t0, *t1).
void group_range(const Plan& p, const GroupedLayout& g, size_t i, int c0, int c1, int64_t* s0, int64_t* s1,
                 int64_t* t0, int64_t* t1) {
  const int l = g.hl[i];
  const int64_t f = g.fl[i];
  *s0 = p.sS.cone_begin[l][c0 * f];
  *s1 = p.sS.cone_begin[l][c1 * f];
  *t0 = p.sT.cone_begin[l][c0 * f];
  *t1 = p.sT.cone_begin[l][c1 * f];
}

// Grouped layout for R right-hand sides per pass: the HF levels split into
// direction groups that fit the device memory (or `groups_forced` groups),
// one group's M and L at a time, LF levels resident.
int prepare_grouped(defmm_handle* h, int R) {
  if (h->layout == 2 && h->gl.R == R) return 0;
  drop_graph(h);
  free_buf(h->M);
  free_buf(h->Lx);
  free_buf(h->F);
  free_buf(h->q);
  free_buf(h->pscr);
  h->use_sym = false;
  free_grouped(h);
  h->layout = 0;
  Plan& p = h->plan;
  GroupedLayout& g = h->gl;
  g.R = R;
  const bool fp64 = h->precision == DEFMM_PRECISION_FP64;
  const size_t cs = fp64 ? 16 : 8;
  const Levels& v = p.lv;
  // HF levels with slots (contiguous, coarse to fine) and the pivot
  for (int l = 0; l < v.nlvl; l++)
    if (v.prec[l] && v.isHF[l] && p.sS.lvl_begin[l + 1] + p.sT.lvl_begin[l + 1] > p.sS.lvl_begin[l] + p.sT.lvl_begin[l])
      g.hl.push_back(l);
  for (size_t i = 1; i < g.hl.size(); i++)
    if (g.hl[i] != g.hl[i - 1] + 1) return h->fail(DEFMM_ERR_ARG, "grouped layout: HF levels are not contiguous");
  g.lh = g.hl.empty() ? -1 : g.hl.back();
  for (int l : g.hl) g.fl.push_back((int64_t)1 << (2 * (v.HFStage[l] - v.HFStage[g.lh])));
  // LF slots: every level below the pivot (or every level without HF slots)
  const int lf = g.lh < 0 ? 0 : g.lh + 1;
  g.lfS0 = p.sS.lvl_begin[lf];
  g.lfS1 = p.sS.n;
  g.lfT0 = p.sT.lvl_begin[lf];
  g.lfT1 = p.sT.n;
  const int64_t nS = (int64_t)p.S.perm.size(), nT = (int64_t)p.T.perm.size();
  const size_t slot_b = (size_t)R * p.LL * cs;
  const size_t nitem = (size_t)std::max<int64_t>(1, p.near_items());
  int st;
  if ((st = ensure(h, g.q, (size_t)nS * R * cs)) || (st = ensure(h, g.pnear, (size_t)nT * R * 16)) ||
      (st = ensure(h, g.pfar, (size_t)nT * R * 16)) || (st = ensure(h, g.tpart, nitem * 32 * R * 16)) ||
      (st = ensure(h, g.Mlf, std::max<int64_t>(1, g.lfS1 - g.lfS0) * slot_b)) ||
      (st = ensure(h, g.Llf, std::max<int64_t>(1, g.lfT1 - g.lfT0) * slot_b)))
    return st;
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  // F batch: at least the largest cone, at most a quarter of the free memory
  // (and 32 GB)
  const size_t fper = (size_t)R * p.PP * cs;
  const int64_t need = largest_cone(p);
  int64_t cap = (int64_t)(std::min<size_t>(fr / 4, (size_t)32 << 30) / fper);
  int64_t want = 0;
  for (int l = 0; l < v.nlvl; l++) want = std::max(want, p.sS.cone_begin[l].back() - p.sS.cone_begin[l].front());
  cap = std::min(cap, std::max(want, need));
  if (cap < need) return h->fail(DEFMM_ERR_MEMORY, "not enough device memory for one cone of spectra");
  g.f_cap = cap;
  if ((st = ensure(h, g.F, (size_t)cap * fper + 16))) return st;  // slack for 16-byte-rounded bulk copies
  // direction groups: consecutive pivot directions while the group's M and L
  // fit in 70% of what is left (or about 1 / groups_forced of all HF slots)
  if (g.lh >= 0) {
    CK(cudaMemGetInfo(&fr, &tot));
    const int nd = v.nDir[g.lh];
    std::vector<int64_t> cost(nd, 0), cS(nd, 0), cT(nd, 0);
    int64_t total = 0;
    for (int c = 0; c < nd; c++) {
      for (size_t i = 0; i < g.hl.size(); i++) {
        int64_t s0, s1, t0, t1;
        group_range(p, g, i, c, c + 1, &s0, &s1, &t0, &t1);
        cS[c] += s1 - s0;
        cT[c] += t1 - t0;
      }
      cost[c] = cS[c] + cT[c];
      total += cost[c];
    }
    int64_t budget = (int64_t)(0.7 * (double)fr / (double)slot_b);
    if (h->groups_forced > 0) budget = std::max<int64_t>(1, (total + h->groups_forced - 1) / h->groups_forced);
    int c0 = 0;
    while (c0 < nd) {
      int c1 = c0 + 1;
      int64_t acc = cost[c0];
      while (c1 < nd && acc + cost[c1] <= budget) acc += cost[c1++];
      int64_t gs = 0, gt = 0;
      for (int c = c0; c < c1; c++) {
        gs += cS[c];
        gt += cT[c];
      }
      g.gS_max = std::max(g.gS_max, gs);
      g.gT_max = std::max(g.gT_max, gt);
      g.groups.push_back({c0, c1});
      c0 = c1;
    }
    if ((st = ensure(h, g.Mg, std::max<int64_t>(1, g.gS_max) * slot_b)) ||
        (st = ensure(h, g.Lg, std::max<int64_t>(1, g.gT_max) * slot_b)))
      return st;
  }
  h->layout = 2;
  return 0;
}

// Tensor-core leaf interpolation in use: requested, and an order whose
// 3-pass split-TF32 GEMMs keep the mixed path within 1e-6 of FP64 (at order
// 8 the equispaced bases' cancellation needs more than the ~22 bits of a
// TF32 pair: CUDA-core FP32 there).
bool tc_on(const defmm_handle* h) { return h->use_tc && h->plan.L <= 7; }

void rec(defmm_handle* h, int i) {
  if (h->events) cudaEventRecord(h->ev[i], h->cur);
}

// One matvec, everything on the device: qin (user order) -> out (user order).
int run_gemv(defmm_handle* h, const double2* qin, double2* out, cudaStream_t s) {
  Plan& p = h->plan;
  const bool fp64 = h->precision == DEFMM_PRECISION_FP64;
  const DevPlan& d = h->dp;
  const dfb::OpTable* ops = h->ops;
  const int64_t nS = (int64_t)p.S.perm.size(), nT = (int64_t)p.T.perm.size();
  const int nl = p.lv.nlvl;
  h->cur = s;
  int64_t nl_ = 0;
  // autotuner timing run: only the phases its choices change (the near
  // field, and M2L of the level with the most far pairs) on whatever the
  // buffers hold; the next full matvec starts from fresh gathers and zeros
  const bool tuning = h->tune_level >= 0 && h->events;
  rec(h, 2 * PH_TOTAL);
  if (!tuning) {
    dfb::launch_gather(fp64, qin, d.S_perm, h->q.p, nS, 0, 0, 1, s);
    nl_ += 1 + (p.p2m_leaf.empty() ? 0 : 1) + (p.l2p_leaf.empty() ? 0 : 1) + 1;
    CK(cudaMemsetAsync(h->pfar.p, 0, 16 * nT, s));
    CK(cudaMemsetAsync(h->Lx.p, 0, h->Lx.bytes, s));
  }
  CK(cudaMemsetAsync(h->pnear.p, 0, 16 * nT, s));
  // near field on the second stream, overlapping the far field
  // (profiling runs it on the main stream so that phase times do not overlap)
  cudaStream_t sn = h->events ? s : h->st2;
  const cudaStream_t sf = s;
  cudaEvent_t ready = h->ev_ready;
  CK(cudaEventRecord(ready, s));
  CK(cudaStreamWaitEvent(sn, ready, 0));
  if (h->events) cudaEventRecord(h->ev[2 * PH_P2P], sn);
  if (h->use_sym) {  // own leaves, then symmetric blocks, then the mirrored partial sums
    dfb::launch_p2p(fp64, d, p.near_self_items(), h->d_self_order, nullptr, h->d_tfirst, h->d_tn,
                    h->d_self_ptr, h->d_self_sfirst, h->d_self_sn, h->q.p, (double2*)h->pnear.p, nullptr,
                    h->d_queue, h->nsm, sn);
    dfb::launch_p2p_sym(fp64, d, p.near_sym_items(), h->d_sym_order, h->d_sym_item_chunk, h->d_tfirst,
                        h->d_tn, h->d_sym_ptr, h->d_sym_sfirst, h->d_sym_sn, h->d_sym_soff, h->q.p, h->d_tpart,
                        h->pscr.p, h->d_queue, h->nsm, h->p2p_bps[fp64 ? 0 : 1], sn);
    dfb::launch_p2p_items(h->nchunk, h->d_tfirst, h->d_tn, h->d_sym_chunk_items, h->d_tpart, (double2*)h->pnear.p,
                          h->nsm, sn);
    dfb::launch_p2p_reduce(fp64, p.near_red_leaves(), h->d_red_first, h->d_red_n, h->d_red_ptr,
                           h->d_red_off, h->pscr.p, (double2*)h->pnear.p, h->nsm, sn);
    nl_ += (p.near_self_items() ? 1 : 0) + (p.near_sym_items() ? 2 : 0) + (p.near_red_leaves() ? 1 : 0);
  } else {  // every interaction from the target side, in items
    dfb::launch_p2p(fp64, d, p.near_items(), h->d_p2p_order, h->d_p2p_item_chunk, h->d_tfirst, h->d_tn,
                    h->d_p2p_ptr, h->d_sfirst, h->d_sn, h->q.p, (double2*)h->pnear.p, h->d_tpart, h->d_queue,
                    h->nsm, sn);
    dfb::launch_p2p_items(h->nchunk, h->d_tfirst, h->d_tn, h->d_p2p_chunk_items, h->d_tpart, (double2*)h->pnear.p,
                          h->nsm, sn);
    nl_ += p.near_items() ? 2 : 0;
  }
  if (h->events) cudaEventRecord(h->ev[2 * PH_P2P + 1], sn);
  if (tuning) {
    // M2L candidates on interleaved slices of each tuned level's target
    // slots (slice i runs candidate i mod 4), timed per slice and counted in
    // far pairs, so one run compares every candidate on every tuned level
    float tm2l = 0;
    for (int l = p.lv.max_stage; l < nl && h->tune_m2l; l++) {
      for (int c = 0; c < 4; c++) h->tune_ms[l][c] = h->tune_pairs[l][c] = 0;
      if (!h->tune_lvl_on[l]) continue;
      const auto& cS = p.sS.cone_begin[l];
      const auto& cT = p.sT.cone_begin[l];
      const int nc = (int)cS.size() - 1;
      for (int c0 = 0; c0 < nc;) {
        int c1 = c0 + 1;
        while (c1 < nc && cS[c1 + 1] - cS[c0] <= h->f_cap) c1++;
        const int64_t fs0 = cS[c0], fs1 = cS[c1], ts0 = cT[c0], ts1 = cT[c1];
        constexpr int kSlices = 16;
        for (int i = 0; i < kSlices && ts1 > ts0 && fs1 > fs0; i++) {
          const int64_t a0 = ts0 + (ts1 - ts0) * i / kSlices, a1 = ts0 + (ts1 - ts0) * (i + 1) / kSlices;
          if (a1 <= a0) continue;
          const int c = i % 4;
          rec(h, 2 * PH_M2L);
          ops->m2l(d, a0, a1, fs0, fs1, h->F.p, h->ptab.p, h->Lx.p, h->d_queue + 1, h->nsm, kM2LCand[c][1],
                   kM2LCand[c][0], sf);
          rec(h, 2 * PH_M2L + 1);
          nl_++;
          float a;
          CK(cudaEventSynchronize(h->ev[2 * PH_M2L + 1]));
          cudaEventElapsedTime(&a, h->ev[2 * PH_M2L], h->ev[2 * PH_M2L + 1]);
          tm2l += a;
          h->tune_ms[l][c] += a;
          h->tune_pairs[l][c] += (double)(p.m2l_ptr[a1] - p.m2l_ptr[a0]);
        }
        c0 = c1;
      }
    }
    CK(cudaStreamSynchronize(sn));
    CK(cudaStreamSynchronize(s));
    for (int i = 0; i < PH_N; i++) h->phase_ms[i] = 0;
    float a = 0;
    cudaEventElapsedTime(&a, h->ev[2 * PH_P2P], h->ev[2 * PH_P2P + 1]);
    h->phase_ms[PH_P2P] = a;
    h->phase_ms[PH_M2L] = tm2l;
    h->launches += nl_;
    CK(cudaGetLastError());
    return 0;
  }
  // upward pass
  rec(h, 2 * PH_P2M);
  if (!fp64 && tc_on(h))
    dfb::launch_p2m_tc(p.L, d, h->d_p2m_leaf, (int)p.p2m_leaf.size(), h->q.p, h->sig2.p, h->M.p, 1, INT_MIN,
                       INT_MAX, h->nsm, sf);
  else
    ops->p2m(d, h->d_p2m_leaf, (int)p.p2m_leaf.size(), h->q.p, h->sig2.p, h->M.p, 1, INT_MIN, INT_MAX, sf);
  rec(h, 2 * PH_P2M + 1);
  rec(h, 2 * PH_M2M);
  for (int l = nl - 2; l >= p.lv.max_stage; l--) {
    ops->m2m(d, p.sS.lvl_begin[l], p.sS.lvl_begin[l + 1], h->sig.p, h->sig2.p, h->M.p, h->M.p, 1, sf);
    nl_ += p.sS.lvl_begin[l + 1] > p.sS.lvl_begin[l] ? 1 : 0;
  }
  rec(h, 2 * PH_M2M + 1);
  // far field per level and cone batch, then the downward transfer
  float tm2f = 0, tm2l = 0, tl2l = 0;
  const size_t cs = fp64 ? 16 : 8;
  for (int l = p.lv.max_stage; l < nl; l++) {
    const auto& cS = p.sS.cone_begin[l];
    const auto& cT = p.sT.cone_begin[l];
    const int nc = (int)cS.size() - 1;
    int c0 = 0;
    while (c0 < nc) {
      int c1 = c0 + 1;
      while (c1 < nc && cS[c1 + 1] - cS[c0] <= h->f_cap) c1++;
      const int64_t fs0 = cS[c0], fs1 = cS[c1], ts0 = cT[c0], ts1 = cT[c1];
      if (ts1 > ts0 && fs1 > fs0) {
        rec(h, 2 * PH_M2F);
        ops->m2f(fs1 - fs0, (const char*)h->M.p + fs0 * p.LL * cs, h->F.p, sf);
        nl_ += 2;
        rec(h, 2 * PH_M2F + 1);
        rec(h, 2 * PH_M2L);
        int nt_l, pair_l;
        m2l_choice(h, fp64 ? 0 : 1, l, &nt_l, &pair_l);
        ops->m2l(d, ts0, ts1, fs0, fs1, h->F.p, h->ptab.p, h->Lx.p, h->d_queue + 1, h->nsm, nt_l, pair_l, sf);
        rec(h, 2 * PH_M2L + 1);
        if (h->events) {
          float a;
          CK(cudaEventSynchronize(h->ev[2 * PH_M2L + 1]));
          cudaEventElapsedTime(&a, h->ev[2 * PH_M2F], h->ev[2 * PH_M2F + 1]);
          tm2f += a;
          cudaEventElapsedTime(&a, h->ev[2 * PH_M2L], h->ev[2 * PH_M2L + 1]);
          tm2l += a;
        }
      }
      c0 = c1;
    }
    if (l + 1 < nl) {
      rec(h, 2 * PH_L2L);
      ops->l2l(d, p.sT.lvl_begin[l + 1], p.sT.lvl_begin[l + 2], h->sig.p, h->sig2.p, h->Lx.p, h->Lx.p, 1, INT64_MIN,
               INT64_MAX, sf);
      nl_ += p.sT.lvl_begin[l + 2] > p.sT.lvl_begin[l + 1] ? 1 : 0;
      rec(h, 2 * PH_L2L + 1);
      if (h->events) {
        float a;
        CK(cudaEventSynchronize(h->ev[2 * PH_L2L + 1]));
        cudaEventElapsedTime(&a, h->ev[2 * PH_L2L], h->ev[2 * PH_L2L + 1]);
        tl2l += a;
      }
    }
  }
  rec(h, 2 * PH_L2P);
  if (!fp64 && tc_on(h) && h->l2p_max_points <= 128)
    dfb::launch_l2p_tc(p.L, d, h->d_l2p_leaf, (int)p.l2p_leaf.size(), h->sig2.p, h->Lx.p, (double2*)h->pfar.p, 1,
                       INT_MIN, INT_MAX, false, h->nsm, sf);
  else
    ops->l2p(d, h->d_l2p_leaf, (int)p.l2p_leaf.size(), h->sig2.p, h->Lx.p, (double2*)h->pfar.p, 1, INT_MIN, INT_MAX,
             false, sf);
  rec(h, 2 * PH_L2P + 1);
  CK(cudaEventRecord(h->ev_done, sn));
  CK(cudaStreamWaitEvent(s, h->ev_done, 0));
  rec(h, 2 * PH_SCATTER);
  dfb::launch_scatter((const double2*)h->pnear.p, (const double2*)h->pfar.p, d.T_perm, out, nT, s);
  rec(h, 2 * PH_SCATTER + 1);
  rec(h, 2 * PH_TOTAL + 1);
  h->launches += nl_;
  CK(cudaGetLastError());
  if (h->events) {
    CK(cudaStreamSynchronize(s));
    auto el = [&](int ph) {
      float a = 0;
      cudaEventElapsedTime(&a, h->ev[2 * ph], h->ev[2 * ph + 1]);
      return (double)a;
    };
    for (int i = 0; i < PH_N; i++) h->phase_ms[i] = 0;
    h->phase_ms[PH_P2M] = el(PH_P2M);
    h->phase_ms[PH_M2M] = el(PH_M2M);
    h->phase_ms[PH_M2F] = tm2f;
    h->phase_ms[PH_M2L] = tm2l;
    h->phase_ms[PH_F2L] = 0.;  // fused into M2L
    h->phase_ms[PH_L2L] = tl2l;
    h->phase_ms[PH_L2P] = el(PH_L2P);
    h->phase_ms[PH_P2P] = el(PH_P2P);
    h->phase_ms[PH_SCATTER] = el(PH_SCATTER);
    h->phase_ms[PH_TOTAL] = el(PH_TOTAL);
  }
  return 0;
}

// Address of global slot `slot` (right-hand side 0) in a buffer that holds
// the slots [first, ...) with slot_b bytes per slot, as a base for the
// kernels (base + slot * R * LL elements); computed in integers because the
// base itself may lie before the buffer.
void* slot_base(void* buf, int64_t first, size_t slot_b) {
  return reinterpret_cast<void*>(reinterpret_cast<uintptr_t>(buf) - (uintptr_t)((size_t)first * slot_b));
}

// Up to R matvecs in one pass over the grouped layout: qin holds nvec <= R
// user-order charge vectors (vector r at qin + r * stride_in), out receives
// nvec potential vectors (at out + r * stride_out).
int run_gemv_grouped(defmm_handle* h, const double2* qin, int64_t stride_in, double2* out, int64_t stride_out,
                     int nvec, cudaStream_t s) {
  Plan& p = h->plan;
  GroupedLayout& g = h->gl;
  const int R = g.R;
  const bool fp64 = h->precision == DEFMM_PRECISION_FP64;
  const DevPlan& d = h->dp;
  const dfb::OpTable* ops = h->ops;
  const Levels& v = p.lv;
  const int64_t nS = (int64_t)p.S.perm.size(), nT = (int64_t)p.T.perm.size();
  const int nl = v.nlvl;
  const size_t cs = fp64 ? 16 : 8;
  const size_t slot_b = (size_t)R * p.LL * cs;
  const int pi = fp64 ? 0 : 1;
  h->cur = s;
  int64_t nk = 0;  // kernels launched
  for (int i = 0; i < PH_N; i++) h->phase_ms[i] = 0;
  // profiling: each phase segment timed with events on the main stream
  cudaEvent_t e0 = h->ev[0], e1 = h->ev[1];
  auto timed = [&](int ph, auto&& fn) -> int {
    if (h->events) CK(cudaEventRecord(e0, s));
    fn();
    if (h->events) {
      CK(cudaEventRecord(e1, s));
      CK(cudaEventSynchronize(e1));
      float a = 0;
      cudaEventElapsedTime(&a, e0, e1);
      h->phase_ms[ph] += a;
    }
    return 0;
  };
  cudaEvent_t t_all0 = h->ev[2], t_all1 = h->ev[3];
  if (h->events) CK(cudaEventRecord(t_all0, s));
  dfb::launch_gather_rhs(fp64, qin, d.S_perm, g.q.p, nS, stride_in, R, nvec, s);
  nk++;
  CK(cudaMemsetAsync(g.pfar.p, 0, (size_t)nT * R * 16, s));
  CK(cudaMemsetAsync(g.pnear.p, 0, (size_t)nT * R * 16, s));
  if (g.lfT1 > g.lfT0) CK(cudaMemsetAsync(g.Llf.p, 0, (size_t)(g.lfT1 - g.lfT0) * slot_b, s));
  // near field on the second stream (the main one when profiling)
  cudaStream_t sn = h->events ? s : h->st2;
  CK(cudaEventRecord(h->ev_ready, s));
  CK(cudaStreamWaitEvent(sn, h->ev_ready, 0));
  {
    float a = 0;
    if (h->events) CK(cudaEventRecord(e0, sn));
    dfb::launch_p2p_rhs(fp64, d, p.near_items(), h->d_p2p_order, h->d_p2p_item_chunk, h->d_tfirst,
                        h->d_tn, h->d_p2p_ptr, h->d_sfirst, h->d_sn, g.q.p, R, (double2*)g.pnear.p,
                        (double2*)g.tpart.p, h->d_queue, h->nsm, h->p2p_bps[pi], sn);
    dfb::launch_p2p_items_rhs(h->nchunk, h->d_tfirst, h->d_tn, h->d_p2p_chunk_items, (const double2*)g.tpart.p, R,
                              (double2*)g.pnear.p, h->nsm, sn);
    nk += p.near_items() ? (R + 7) / 8 + 1 : 0;
    if (h->events) {
      CK(cudaEventRecord(e1, sn));
      CK(cudaEventSynchronize(e1));
      cudaEventElapsedTime(&a, e0, e1);
      h->phase_ms[PH_P2P] += a;
    }
  }
  // P2M of the given leaves' slots with directions in [d0, d1) into Mbase
  auto p2m = [&](const int32_t* leaves, int n, void* Mbase, int d0, int d1) {
    if (!fp64 && tc_on(h))
      dfb::launch_p2m_tc(p.L, d, leaves, n, g.q.p, h->sig2.p, Mbase, R, d0, d1, h->nsm, s);
    else
      ops->p2m(d, leaves, n, g.q.p, h->sig2.p, Mbase, R, d0, d1, s);
  };
  // L2P of the given leaves' slots with directions in [d0, d1) from Lbase
  auto l2p = [&](const int32_t* leaves, int n, const void* Lbase, int d0, int d1) {
    if (!fp64 && tc_on(h) && h->l2p_max_points <= 128)
      dfb::launch_l2p_tc(p.L, d, leaves, n, h->sig2.p, Lbase, (double2*)g.pfar.p, R, d0, d1, true, h->nsm, s);
    else
      ops->l2p(d, leaves, n, h->sig2.p, Lbase, (double2*)g.pfar.p, R, d0, d1, true, s);
  };
  void* Mlf = slot_base(g.Mlf.p, g.lfS0, slot_b);
  void* Llf = slot_base(g.Llf.p, g.lfT0, slot_b);
  const int lf = g.lh < 0 ? 0 : g.lh + 1;  // first LF level
  // M2F + M2L of source cones [c0, c1) at level l: targets into Lbase
  auto far_cones = [&](int l, int64_t c0, int64_t c1, void* Mbase, void* Lbase) -> int {
    const auto& cS = p.sS.cone_begin[l];
    const auto& cT = p.sT.cone_begin[l];
    int64_t a = c0;
    while (a < c1) {
      int64_t b = a + 1;
      while (b < c1 && cS[b + 1] - cS[a] <= g.f_cap) b++;
      const int64_t fs0 = cS[a], fs1 = cS[b], ts0 = cT[a], ts1 = cT[b];
      if (ts1 > ts0 && fs1 > fs0) {
        timed(PH_M2F, [&] {
          ops->m2f((fs1 - fs0) * R, (const char*)Mbase + (size_t)fs0 * slot_b, g.F.p, s);
        });
        timed(PH_M2L, [&] {
          if (R == 1) {
            int nt_l, pair_l;
            m2l_choice(h, pi, l, &nt_l, &pair_l);
            ops->m2l(d, ts0, ts1, fs0, fs1, g.F.p, h->ptab.p, Lbase, h->d_queue + 1, h->nsm, nt_l, pair_l, s);
          } else
            ops->m2l_rhs(d, ts0, ts1, fs0, fs1, R, h->rhs_block_m2l, g.F.p, h->ptab.p, Lbase, h->d_queue + 1,
                         h->nsm, h->m2l_staging ? h->m2l_lgroup : 0, s);
        });
        nk += 2;
      }
      a = b;
    }
    return 0;
  };
  // ---- LF levels (resident): upward pass and their far field
  if (g.lfS1 > g.lfS0 || g.lfT1 > g.lfT0) {
    timed(PH_P2M, [&] {
      for (int l = lf; l < nl; l++) {
        const int64_t b = h->p2m_lvl_off[l], e = h->p2m_lvl_off[l + 1];
        if (e > b) {
          p2m(h->d_p2m_bylvl + b, (int)(e - b), Mlf, INT_MIN, INT_MAX);
          nk++;
        }
      }
    });
    timed(PH_M2M, [&] {
      for (int l = nl - 2; l >= lf; l--)
        if (p.sS.lvl_begin[l + 1] > p.sS.lvl_begin[l]) {
          ops->m2m(d, p.sS.lvl_begin[l], p.sS.lvl_begin[l + 1], h->sig.p, h->sig2.p, Mlf, Mlf, R, s);
          nk++;
        }
    });
    for (int l = lf; l < nl; l++)
      if (v.prec[l]) far_cones(l, 0, (int64_t)p.sS.cone_begin[l].size() - 1, Mlf, Llf);
  }
  // ---- HF levels, one direction group at a time
  h->groups_used = (int)g.groups.size();
  for (const auto& gr : g.groups) {
    const int c0 = gr.first, c1 = gr.second;
    const size_t nh = g.hl.size();
    std::vector<int64_t> s0(nh), s1(nh), t0(nh), t1(nh);
    std::vector<void*> Mb(nh), Lb(nh);
    int64_t so = 0, to = 0;
    for (size_t i = 0; i < nh; i++) {
      group_range(p, g, i, c0, c1, &s0[i], &s1[i], &t0[i], &t1[i]);
      Mb[i] = slot_base((char*)g.Mg.p + (size_t)so * slot_b, s0[i], slot_b);
      Lb[i] = slot_base((char*)g.Lg.p + (size_t)to * slot_b, t0[i], slot_b);
      so += s1[i] - s0[i];
      to += t1[i] - t0[i];
    }
    if (to > 0) CK(cudaMemsetAsync(g.Lg.p, 0, (size_t)to * slot_b, s));
    // upward: P2M of the group's leaf slots, M2M level by level
    timed(PH_P2M, [&] {
      for (size_t i = 0; i < nh; i++) {
        const int l = g.hl[i];
        const int64_t b = h->p2m_lvl_off[l], e = h->p2m_lvl_off[l + 1];
        if (e > b && s1[i] > s0[i]) {
          p2m(h->d_p2m_bylvl + b, (int)(e - b), Mb[i], (int)(c0 * g.fl[i]), (int)(c1 * g.fl[i]));
          nk++;
        }
      }
    });
    timed(PH_M2M, [&] {
      for (int i = (int)nh - 1; i >= 0; i--) {
        if (s1[i] <= s0[i]) continue;
        const void* Mc = (size_t)i + 1 < nh ? Mb[i + 1] : Mlf;  // children: next HF level or the LF level below
        ops->m2m(d, s0[i], s1[i], h->sig.p, h->sig2.p, Mb[i], Mc, R, s);
        nk++;
      }
    });
    // far field top-down, then the downward transfer
    for (size_t i = 0; i < nh; i++) {
      far_cones(g.hl[i], (int64_t)c0 * g.fl[i], (int64_t)c1 * g.fl[i], Mb[i], Lb[i]);
      timed(PH_L2L, [&] {
        if (i + 1 < nh) {
          if (t1[i + 1] > t0[i + 1]) {
            ops->l2l(d, t0[i + 1], t1[i + 1], h->sig.p, h->sig2.p, Lb[i + 1], Lb[i], R, t0[i], t1[i], s);
            nk++;
          }
        } else if (g.hl[i] + 1 < nl) {  // into the LF level below, from this group's parents only
          const int l = g.hl[i] + 1;
          if (p.sT.lvl_begin[l + 1] > p.sT.lvl_begin[l]) {
            ops->l2l(d, p.sT.lvl_begin[l], p.sT.lvl_begin[l + 1], h->sig.p, h->sig2.p, Llf, Lb[i], R, t0[i], t1[i],
                     s);
            nk++;
          }
        }
      });
    }
    timed(PH_L2P, [&] {
      for (size_t i = 0; i < nh; i++) {
        const int l = g.hl[i];
        const int64_t b = h->l2p_lvl_off[l], e = h->l2p_lvl_off[l + 1];
        if (e > b && t1[i] > t0[i]) {
          l2p(h->d_l2p_bylvl + b, (int)(e - b), Lb[i], (int)(c0 * g.fl[i]), (int)(c1 * g.fl[i]));
          nk++;
        }
      }
    });
  }
  // ---- LF levels: downward pass and L2P
  if (g.lfT1 > g.lfT0) {
    timed(PH_L2L, [&] {
      for (int l = lf; l + 1 < nl; l++)
        if (p.sT.lvl_begin[l + 2] > p.sT.lvl_begin[l + 1]) {
          ops->l2l(d, p.sT.lvl_begin[l + 1], p.sT.lvl_begin[l + 2], h->sig.p, h->sig2.p, Llf, Llf, R, INT64_MIN,
                   INT64_MAX, s);
          nk++;
        }
    });
    timed(PH_L2P, [&] {
      for (int l = lf; l < nl; l++) {
        const int64_t b = h->l2p_lvl_off[l], e = h->l2p_lvl_off[l + 1];
        if (e > b) {
          l2p(h->d_l2p_bylvl + b, (int)(e - b), Llf, INT_MIN, INT_MAX);
          nk++;
        }
      }
    });
  }
  CK(cudaEventRecord(h->ev_done, sn));
  CK(cudaStreamWaitEvent(s, h->ev_done, 0));
  timed(PH_SCATTER, [&] {
    dfb::launch_scatter_rhs((const double2*)g.pnear.p, (const double2*)g.pfar.p, d.T_perm, out, nT, stride_out, R,
                            nvec, s);
  });
  nk++;
  if (h->events) {
    CK(cudaEventRecord(t_all1, s));
    CK(cudaEventSynchronize(t_all1));
    float a = 0;
    cudaEventElapsedTime(&a, t_all0, t_all1);
    h->phase_ms[PH_TOTAL] = a;
  }
  h->launches += nk;
  CK(cudaGetLastError());
  return 0;
}

// Device bytes held by the expansion layout of the current precision.
size_t layout_bytes(const defmm_handle* h) {
  const GroupedLayout& g = h->gl;
  size_t b = h->M.bytes + h->Lx.bytes + h->F.bytes + h->q.bytes + h->pscr.bytes;
  for (const DevBuf* x : {&g.Mg, &g.Lg, &g.Mlf, &g.Llf, &g.F, &g.q, &g.pnear, &g.pfar, &g.tpart}) b += x->bytes;
  return b;
}

// Right-hand sides per pass of the grouped layout for a call with nrhs
// right-hand sides, or 0 for the resident layout (one right-hand side whose
// M and L of every slot fit in 85% of the memory this handle can use).
int choose_rhs_block(defmm_handle* h, int64_t nrhs) {
  if (nrhs > 1) return (int)std::min<int64_t>(std::max(1, h->rhs_block), nrhs);
  if (h->groups_forced > 0) return 1;
  if (h->layout == 1) return 0;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return (double)resident_bytes(h) <= 0.85 * (double)(fr + layout_bytes(h)) ? 0 : 1;
}

// nrhs matvecs on device vectors (rhs-major, user order) through the grouped
// layout with R right-hand sides per pass.
int gemv_grouped(defmm_handle* h, const double2* in, double2* out, int64_t nrhs, int R, cudaStream_t s) {
  int st = prepare_grouped(h, R);
  if (st) return st;
  const int64_t nS = (int64_t)h->plan.S.perm.size(), nT = (int64_t)h->plan.T.perm.size();
  for (int64_t b = 0; b < nrhs; b += R) {
    const int nvec = (int)std::min<int64_t>(R, nrhs - b);
    st = run_gemv_grouped(h, in + b * nS, nS, out + b * nT, nT, nvec, s);
    if (st) return st;
  }
  return 0;
}

// One matvec on stream s, replaying a captured graph when possible.
int matvec(defmm_handle* h, const double2* qin, double2* out, cudaStream_t s) {
  if (!h->use_graphs || h->events) return run_gemv(h, qin, out, s);
  if (h->gexec && h->g_in == qin && h->g_out == out && h->g_stream == s && h->g_prec == h->precision) {
    CK(cudaGraphLaunch(h->gexec, s));
    h->launches += h->g_launches;
    return 0;
  }
  drop_graph(h);
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const int64_t before = h->launches;
  int st = run_gemv(h, qin, out, s);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (st) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->use_graphs = false;  // capture not possible here: run directly from now on
    return run_gemv(h, qin, out, s);
  }
  e = cudaGraphInstantiate(&h->gexec, g, 0);
  h->graph = g;  // kept: batches embed it as a child graph
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->gexec = nullptr;
    h->use_graphs = false;
    return run_gemv(h, qin, out, s);
  }
  h->g_in = qin;
  h->g_out = out;
  h->g_stream = s;
  h->g_prec = h->precision;
  h->g_launches = h->launches - before;
  CK(cudaGraphLaunch(h->gexec, s));
  return 0;
}

int ensure_device(defmm_handle* h) {
  if (h->device >= 0) return 0;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return h->fail(DEFMM_ERR_CUDA, "no CUDA device available");
  }
  CK(cudaGetDevice(&h->device));
  CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&h->st2, cudaStreamNonBlocking));
  for (int i = 0; i < 2 * PH_N; i++) CK(cudaEventCreate(&h->ev[i]));
  CK(cudaEventCreateWithFlags(&h->ev_ready, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ev_qin_read, cudaEventDisableTiming));
  return 0;
}

// Launch choices of defmm_autotune per operator shape (order, precision,
// levels, slots, far pairs, particle interactions, device) in this process.
std::mutex g_tune_mu;
struct TuneChoice {
  int nt = 128, pair = 0, bps = 16;
  int16_t lvl_nt[32], lvl_pair[32];  // per level; < 0: nt / pair
};
std::map<std::array<int64_t, 9>, TuneChoice> g_tune;

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

}  // namespace

// ==================================================================== C ABI
extern "C" {

int defmm_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

defmm_handle* defmm_create(void) {
  defmm_handle* h = new defmm_handle();
  m2l_levels_reset(h, 0);
  m2l_levels_reset(h, 1);
  return h;
}

void defmm_destroy(defmm_handle* h) {
  if (!h) return;
  if (h->device >= 0) {
    cudaSetDevice(h->device);
    free_plan_device(h);
    for (int i = 0; i < 2 * PH_N; i++)
      if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    if (h->ev_ready) cudaEventDestroy(h->ev_ready);
    if (h->ev_done) cudaEventDestroy(h->ev_done);
    if (h->ev_qin_read) cudaEventDestroy(h->ev_qin_read);
    if (h->st) cudaStreamDestroy(h->st);
    if (h->st2) cudaStreamDestroy(h->st2);
  }
  delete h;
}

const char* defmm_last_error(const defmm_handle* h) { return h ? h->err.c_str() : "null handle"; }

int defmm_add_source_particle(defmm_handle* h, const double xyz[3]) {
  if (!h || !xyz) return DEFMM_ERR_ARG;
  h->src.insert(h->src.end(), xyz, xyz + 3);
  return 0;
}
int defmm_add_target_particle(defmm_handle* h, const double xyz[3]) {
  if (!h || !xyz) return DEFMM_ERR_ARG;
  h->trg.insert(h->trg.end(), xyz, xyz + 3);
  return 0;
}
int defmm_add_sources(defmm_handle* h, const double* xyz, int64_t n) {
  if (!h || (n > 0 && !xyz) || n < 0) return DEFMM_ERR_ARG;
  h->src.insert(h->src.end(), xyz, xyz + 3 * n);
  return 0;
}
int defmm_add_targets(defmm_handle* h, const double* xyz, int64_t n) {
  if (!h || (n > 0 && !xyz) || n < 0) return DEFMM_ERR_ARG;
  h->trg.insert(h->trg.end(), xyz, xyz + 3 * n);
  return 0;
}

int defmm_load_inp(defmm_handle* h, const char* path, int64_t nparts, int which) {
  if (!h || !path || nparts < 0 || (which != 0 && which != 1)) return DEFMM_ERR_ARG;
  FILE* f = std::fopen(path, "r");
  if (!f) return h->fail(DEFMM_ERR_IO, std::string("cannot open ") + path);
  std::vector<double> v(3 * nparts);
  for (int64_t i = 0; i < 3 * nparts; i++)
    if (std::fscanf(f, "%lf", &v[i]) != 1) {
      std::fclose(f);
      return h->fail(DEFMM_ERR_IO, std::string("short INP file ") + path);
    }
  std::fclose(f);
  auto& dst = which == 0 ? h->src : h->trg;
  dst.insert(dst.end(), v.begin(), v.end());
  return 0;
}

int defmm_set_graphs(defmm_handle* h, int on) {
  if (!h) return DEFMM_ERR_ARG;
  h->use_graphs = on != 0;
  if (!h->use_graphs && h->device >= 0) drop_graph(h);
  return 0;
}

int defmm_set_profiling(defmm_handle* h, int on) {
  if (!h) return DEFMM_ERR_ARG;
  h->events = on != 0;
  return 0;
}

int defmm_set_launch(defmm_handle* h, int m2l_threads, int p2p_blocks_per_sm) {
  if (!h || (m2l_threads != 0 && m2l_threads != 128 && m2l_threads != 256) || p2p_blocks_per_sm < 0 ||
      p2p_blocks_per_sm > 64)
    return DEFMM_ERR_ARG;
  const int pi = h->precision == DEFMM_PRECISION_FP64 ? 0 : 1;
  h->m2l_nt[pi] = m2l_threads;
  h->p2p_bps[pi] = p2p_blocks_per_sm ? p2p_blocks_per_sm : 16;
  m2l_levels_reset(h, pi);
  if (h->device >= 0) drop_graph(h);
  return 0;
}

int defmm_set_m2l_pairing(defmm_handle* h, int on) {
  if (!h || (on != 0 && on != 1)) return DEFMM_ERR_ARG;
  h->m2l_pair[h->precision == DEFMM_PRECISION_FP64 ? 0 : 1] = on;
  m2l_levels_reset(h, h->precision == DEFMM_PRECISION_FP64 ? 0 : 1);
  if (h->device >= 0) drop_graph(h);
  return 0;
}

int defmm_autotune(defmm_handle* h, int reps, int32_t* choice) {
  if (!h || reps < 1 || reps > 100) return DEFMM_ERR_ARG;
  if (!h->built) return h->fail(DEFMM_ERR_ARG, "autotune before prcmpt");
  int st = defmm_upload(h);
  if (st) return st;
  // choices already timed on an operator of the same shape in this process
  const Plan& pl = h->plan;
  const std::array<int64_t, 9> key = {pl.L, h->precision, pl.lv.nlvl, pl.sS.n, pl.sT.n, pl.n_far_hf,
                                      pl.n_far_lf, pl.i_near, h->device};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      const int pi = h->precision == DEFMM_PRECISION_FP64 ? 0 : 1;
      const TuneChoice& c = it->second;
      h->m2l_nt[pi] = c.nt;
      h->m2l_pair[pi] = c.pair;
      h->p2p_bps[pi] = c.bps;
      for (int l = 0; l < 32; l++) {
        h->m2l_lvl_nt[pi][l] = c.lvl_nt[l];
        h->m2l_lvl_pair[pi][l] = c.lvl_pair[l];
      }
      drop_graph(h);
      if (choice) {
        choice[0] = c.nt;
        choice[1] = c.bps;
      }
      return 0;
    }
  }
  st = prepare_precision(h);
  if (st) return st;
  const int64_t nS = (int64_t)h->plan.S.perm.size(), nT = (int64_t)h->plan.T.perm.size();
  if ((st = ensure(h, h->rin, 16 * nS)) || (st = ensure(h, h->rout, 16 * nT))) return st;
  CK(cudaMemsetAsync(h->rin.p, 0, 16 * nS, h->st));
  const int pi = h->precision == DEFMM_PRECISION_FP64 ? 0 : 1;
  const bool ev = h->events;
  h->events = true;  // phase timers, phases serialised
  drop_graph(h);     // the captured graph holds the old launch choices
  // timing runs (run_gemv in tuning mode): the near field, and once the M2L
  // of the tuned levels, so each level gets its own launch choice
  const Plan& q = h->plan;
  int busiest = q.lv.max_stage;
  {
    int64_t best = -1;
    for (int l = q.lv.max_stage; l < q.lv.nlvl; l++) {
      const int64_t e = q.m2l_ptr[q.sT.lvl_begin[l + 1]] - q.m2l_ptr[q.sT.lvl_begin[l]];
      if (e > best) {
        best = e;
        busiest = l;
      }
    }
  }
  h->tune_level = busiest;
  m2l_levels_reset(h, pi);
  // levels timed on their own: those with at least 2% of the far pairs (the
  // others take the busiest level's choice)
  {
    const int64_t tot = q.m2l_ptr.empty() ? 0 : q.m2l_ptr.back();
    for (int l = 0; l < 32; l++) h->tune_lvl_on[l] = false;
    for (int l = q.lv.max_stage; l < q.lv.nlvl; l++) {
      const int64_t e = q.m2l_ptr[q.sT.lvl_begin[l + 1]] - q.m2l_ptr[q.sT.lvl_begin[l]];
      h->tune_lvl_on[l] = l == busiest || 50 * e >= tot;
    }
  }
  // three timing runs, one per near-field candidate; the first also times
  // the four M2L candidates (one or two target slots per CTA at 128 or 256
  // threads) on interleaved slices of every tuned level
  int bps_best = 16;
  double tb_p2p = 1e300, tb_lvl[32];
  int best_lvl[32];
  for (int l = 0; l < 32; l++) {
    tb_lvl[l] = 1e300;
    best_lvl[l] = 0;
  }
  const int bps_cand[3] = {8, 16, 32};
  for (int r = 0; r < reps && !st; r++)
    for (int i = 0; i < 3 && !st; i++) {
      h->p2p_bps[pi] = bps_cand[i];
      h->tune_m2l = i == 0;
      st = run_gemv(h, (const double2*)h->rin.p, (double2*)h->rout.p, h->st);
      if (st) break;
      if (h->phase_ms[PH_P2P] < tb_p2p) {
        tb_p2p = h->phase_ms[PH_P2P];
        bps_best = bps_cand[i];
      }
      if (i == 0)
        for (int l = q.lv.max_stage; l < q.lv.nlvl; l++)
          for (int c = 0; c < 4; c++)
            if (h->tune_lvl_on[l] && h->tune_pairs[l][c] > 0) {
              const double t = h->tune_ms[l][c] / h->tune_pairs[l][c];
              if (t < tb_lvl[l]) {
                tb_lvl[l] = t;
                best_lvl[l] = c;
              }
            }
    }
  h->tune_m2l = 0;
  const int (&m2l_cand)[4][2] = kM2LCand;
  // operator-wide choice: the busiest level's; per-level overrides elsewhere
  TuneChoice c;
  c.nt = m2l_cand[best_lvl[busiest]][1];
  c.pair = m2l_cand[best_lvl[busiest]][0];
  c.bps = bps_best;
  for (int l = 0; l < 32; l++) c.lvl_nt[l] = c.lvl_pair[l] = -1;
  for (int l = q.lv.max_stage; l < q.lv.nlvl; l++)
    if (h->tune_lvl_on[l]) {
      c.lvl_nt[l] = (int16_t)m2l_cand[best_lvl[l]][1];
      c.lvl_pair[l] = (int16_t)m2l_cand[best_lvl[l]][0];
    }
  h->m2l_nt[pi] = c.nt;
  h->m2l_pair[pi] = c.pair;
  h->p2p_bps[pi] = c.bps;
  for (int l = 0; l < 32; l++) {
    h->m2l_lvl_nt[pi][l] = c.lvl_nt[l];
    h->m2l_lvl_pair[pi][l] = c.lvl_pair[l];
  }
  h->events = ev;
  h->tune_level = -1;
  if (st) return st;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = c;
  }
  if (choice) {
    choice[0] = c.nt;
    choice[1] = c.bps;
  }
  return 0;
}

int defmm_m2l_schedule(const defmm_handle* h, int32_t* threads, int32_t* pairing, int n) {
  if (!h || n < 0 || (n && (!threads || !pairing))) return DEFMM_ERR_ARG;
  const int pi = h->precision == DEFMM_PRECISION_FP64 ? 0 : 1;
  const int PP = h->built ? h->plan.PP : 0;
  for (int l = 0; l < n; l++) {
    int nt = 0, pair = 0;
    if (l < 32) m2l_choice(h, pi, l, &nt, &pair);
    threads[l] = nt ? nt : (PP > 1024 ? 256 : 128);
    pairing[l] = pair;
  }
  return 0;
}

int defmm_set_plan_device(defmm_handle* h, int on) {
  if (!h) return DEFMM_ERR_ARG;
  h->plan_device = on != 0;
  return 0;
}

int defmm_keep_lists(defmm_handle* h, int on) {
  if (!h) return DEFMM_ERR_ARG;
  h->keep_lists = on != 0;
  return 0;
}

int defmm_prcmpt(defmm_handle* h, int L, int Ncrit, double kappa, int lvMAX) {
  if (!h) return DEFMM_ERR_ARG;
  if (h->src.empty() || h->trg.empty()) return h->fail(DEFMM_ERR_ARG, "no source or no target particles");
  if (!(kappa >= 0.) || !std::isfinite(kappa)) return h->fail(DEFMM_ERR_ARG, "wavenumber must be finite and >= 0");
  if (h->device >= 0) {
    CK(cudaSetDevice(h->device));
    free_plan_device(h);
  }
  h->built = false;
  h->uploaded = false;
  h->plan = Plan();
  h->plan.keep_lists = h->keep_lists;
  std::string e;
  // the level walk on the GPU when there is one (list records for parity
  // checks come from the host walk)
  dfb::LevelWalker* walker = nullptr;
  std::unique_ptr<dfb::TreeSorter> sorter;
  h->walked_on_device = false;
  if (h->plan_device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) == cudaSuccess && n > 0 && ensure_device(h) == 0 &&
        cudaSetDevice(h->device) == cudaSuccess) {
      sorter = dfb::make_device_tree_sorter();
      if (!h->keep_lists) walker = dfb::device_level_walker();
    }
    cudaGetLastError();
    h->err.clear();
  }
  int st = dfb::build_plan(h->plan, h->src.data(), (int64_t)h->src.size() / 3, h->trg.data(),
                           (int64_t)h->trg.size() / 3, L, Ncrit, kappa, lvMAX, e, walker, sorter.get());
  // arrays the walk left on the device belong to this handle's plan (also
  // when the build failed part way)
  for (void* q : {h->plan.dev_m2l_src, h->plan.dev_m2l_tab, h->plan.dev_m2m_ptr, h->plan.dev_m2m_child,
                  h->plan.dev_l2l_ptr, h->plan.dev_l2l_parent, h->plan.dev_cslot_T, h->plan.dev_cdir_T,
                  h->plan.dev_cslot_S, h->plan.dev_cdir_S, h->plan.dev_scell_T, h->plan.dev_sdir_T,
                  h->plan.dev_scell_S, h->plan.dev_sdir_S})
    if (q) h->plan_allocs.push_back(q);
  h->plan_allocs.insert(h->plan_allocs.end(), h->plan.dev_near_allocs.begin(), h->plan.dev_near_allocs.end());
  h->plan.dev_near_allocs.clear();
  if (st) return h->fail(st == -4 ? DEFMM_ERR_CUDA : st == -5 ? DEFMM_ERR_MEMORY : st, e);
  h->walked_on_device = walker != nullptr;
  if (h->plan.lv.nlvl > 32) return h->fail(DEFMM_ERR_DEPTH, "more than 32 tree levels");
  {
    const std::vector<int64_t>& ptr = h->plan.m2l_ptr;
    int64_t lg = 0;
    for (size_t t = 0; t + 1 < ptr.size(); t++)
      lg = std::max(lg, ptr[std::min(ptr.size() - 1, t + dfb::kM2LGroup)] - ptr[t]);
    h->m2l_lgroup = lg;
  }
  h->built = true;
  return 0;
}

int defmm_upload(defmm_handle* h) {
  if (!h) return DEFMM_ERR_ARG;
  if (!h->built) return h->fail(DEFMM_ERR_ARG, "upload before prcmpt");
  int st = ensure_device(h);
  if (st) return st;
  CK(cudaSetDevice(h->device));
  if (h->uploaded) return 0;
  st = upload_plan(h);
  if (st) return st;
  h->uploaded = true;
  return 0;
}

int defmm_set_precision(defmm_handle* h, int mode) {
  if (!h || (mode != DEFMM_PRECISION_FP64 && mode != DEFMM_PRECISION_MIXED)) return DEFMM_ERR_ARG;
  h->precision = mode;
  return 0;
}

int defmm_gemv_device(defmm_handle* h, const void* d_in, void* d_out, int64_t nrhs, void* stream) {
  if (!h || !d_in || !d_out || nrhs < 1) return DEFMM_ERR_ARG;
  if (!h->built) return h->fail(DEFMM_ERR_ARG, "gemv before prcmpt");
  int st = defmm_upload(h);
  if (st) return st;
  st = prepare_tables(h);
  if (st) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : h->st;
  h->launches = 0;
  const int R = choose_rhs_block(h, nrhs);
  if (R > 0) return gemv_grouped(h, (const double2*)d_in, (double2*)d_out, nrhs, R, s);
  st = prepare_resident(h);
  if (st) return st;
  return matvec(h, (const double2*)d_in, (double2*)d_out, s);
}

int defmm_set_blocking(defmm_handle* h, int rhs_block, int groups) {
  if (!h || rhs_block < 1 || rhs_block > dfb::kMaxRhsBlock || groups < 0) return DEFMM_ERR_ARG;
  if (h->rhs_block != rhs_block || h->groups_forced != groups) {
    h->rhs_block = rhs_block;
    h->groups_forced = groups;
    if (h->layout == 2) {  // planned for the old choice
      free_grouped(h);
      h->layout = 0;
    }
  }
  return 0;
}

int defmm_set_tensor_cores(defmm_handle* h, int on) {
  if (!h || (on != 0 && on != 1)) return DEFMM_ERR_ARG;
  if (h->use_tc != (on != 0)) {
    h->use_tc = on != 0;
    if (h->device >= 0) drop_graph(h);
  }
  return 0;
}

int defmm_set_rhs_per_cta(defmm_handle* h, int rb) {
  if (!h || (rb != 1 && rb != 2 && rb != 4 && rb != 8)) return DEFMM_ERR_ARG;
  h->rhs_block_m2l = rb;
  return 0;
}

int defmm_setup_times(const defmm_handle* h, char* buf, int64_t* len) {
  if (!h || !len) return DEFMM_ERR_ARG;
  std::string txt;
  char line[256];
  for (const auto& st : h->plan.t_steps) {
    std::snprintf(line, sizeof(line), "%.6f\t%s\n", st.second, st.first);
    txt += line;
  }
  const int64_t cap = *len;
  *len = (int64_t)txt.size() + 1;
  if (buf && cap > 0) {
    const size_t n = std::min<size_t>((size_t)cap - 1, txt.size());
    std::memcpy(buf, txt.data(), n);
    buf[n] = 0;
  }
  return 0;
}

int defmm_set_m2l_staging(defmm_handle* h, int on) {
  if (!h || (on != 0 && on != 1)) return DEFMM_ERR_ARG;
  h->m2l_staging = on != 0;
  return 0;
}

}  // extern "C"

// Several operators' matvecs as one graph: each handle's captured matvec is
// an independent child node, so independent problems share the GPU.
struct defmm_batch {
  cudaGraphExec_t exec = nullptr;
  int device = -1;
};

extern "C" {

defmm_batch* defmm_batch_create(int64_t n, defmm_handle* const* hs, const void* const* d_in, void* const* d_out,
                                int lanes) {
  if (n < 1 || !hs || !d_in || !d_out || lanes < 1) return nullptr;
  for (int64_t i = 0; i < n; i++)
    if (!hs[i]) return nullptr;
  cudaGraph_t parent = nullptr;
  if (cudaGraphCreate(&parent, 0) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  // longest-first onto the lane with the fewest points so far; within a
  // lane each matvec waits for the previous one
  const int nl = (int)std::min<int64_t>(lanes, n);
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; i++) order[i] = i;
  auto pts = [&](int64_t i) { return (int64_t)(hs[i]->plan.S.perm.size() + hs[i]->plan.T.perm.size()); };
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return pts(a) > pts(b); });
  std::vector<int64_t> load(nl, 0);
  std::vector<cudaGraphNode_t> tail(nl, nullptr);
  int device = -1;
  for (int64_t i : order) {
    defmm_handle* h = hs[i];
    const int lane = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[lane] += pts(i);
    bool ok = h && d_in[i] && d_out[i] && h->built && h->use_graphs;
    // one run on the handle's own stream captures (and runs) its matvec
    if (ok)
      ok = defmm_gemv_device(h, d_in[i], d_out[i], 1, nullptr) == 0 && cudaStreamSynchronize(h->st) == cudaSuccess &&
           h->graph && h->g_in == d_in[i] && h->g_out == d_out[i] && (device < 0 || h->device == device);
    cudaGraphNode_t node;
    if (ok)
      ok = cudaGraphAddChildGraphNode(&node, parent, tail[lane] ? &tail[lane] : nullptr, tail[lane] ? 1 : 0,
                                      h->graph) == cudaSuccess;
    if (ok) tail[lane] = node;
    if (!ok) {
      if (h && h->err.empty()) h->err = "batch: this operator's matvec could not be captured as a graph";
      cudaGetLastError();
      cudaGraphDestroy(parent);
      return nullptr;
    }
    device = h->device;
  }
  defmm_batch* b = new defmm_batch;
  b->device = device;
  cudaError_t e = cudaGraphInstantiate(&b->exec, parent, 0);
  cudaGraphDestroy(parent);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete b;
    return nullptr;
  }
  return b;
}

int defmm_batch_launch(defmm_batch* b, void* stream) {
  if (!b || !b->exec) return DEFMM_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess || cudaGraphLaunch(b->exec, (cudaStream_t)stream) != cudaSuccess) {
    cudaGetLastError();
    return DEFMM_ERR_CUDA;
  }
  return 0;
}

void defmm_batch_destroy(defmm_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  delete b;
}

int defmm_gemv_batched(defmm_handle* h, int64_t nrhs, const double* in, double* out) {
  if (!h || !in || !out || nrhs < 1) return DEFMM_ERR_ARG;
  if (!h->built) return h->fail(DEFMM_ERR_ARG, "gemv before prcmpt");
  int st = defmm_upload(h);
  if (st) return st;
  st = prepare_tables(h);
  if (st) return st;
  const int64_t nS = (int64_t)h->plan.S.perm.size(), nT = (int64_t)h->plan.T.perm.size();
  h->launches = 0;
  // direct sums still reading the previous charges (defmm_direct_noalloc on
  // another stream) finish before qin is overwritten
  CK(cudaStreamWaitEvent(h->st, h->ev_qin_read, 0));
  const int R = choose_rhs_block(h, nrhs);
  if (R == 0) {
    if ((st = prepare_resident(h))) return st;
    for (int64_t r = 0; r < nrhs; r++) {
      CK(cudaMemcpyAsync(h->qin.p, in + 2 * r * nS, 16 * nS, cudaMemcpyHostToDevice, h->st));
      st = matvec(h, (const double2*)h->qin.p, (double2*)h->out.p, h->st);
      if (st) return st;
      CK(cudaMemcpyAsync(out + 2 * r * nT, h->out.p, 16 * nT, cudaMemcpyDeviceToHost, h->st));
    }
  } else {
    // blocks of R right-hand sides staged through the handle's device vectors
    if ((st = prepare_grouped(h, R))) return st;
    if ((st = ensure(h, h->rin, (size_t)16 * nS * R)) || (st = ensure(h, h->rout, (size_t)16 * nT * R))) return st;
    for (int64_t b = 0; b < nrhs; b += R) {
      const int nvec = (int)std::min<int64_t>(R, nrhs - b);
      CK(cudaMemcpyAsync(h->rin.p, in + 2 * b * nS, (size_t)16 * nS * nvec, cudaMemcpyHostToDevice, h->st));
      st = run_gemv_grouped(h, (const double2*)h->rin.p, nS, (double2*)h->rout.p, nT, nvec, h->st);
      if (st) return st;
      CK(cudaMemcpyAsync(out + 2 * b * nT, h->rout.p, (size_t)16 * nT * nvec, cudaMemcpyDeviceToHost, h->st));
    }
    // the last right-hand side's charges and potentials, for the direct-sum checks
    const int last = (int)((nrhs - 1) % R);
    CK(cudaMemcpyAsync(h->qin.p, (const double2*)h->rin.p + (size_t)last * nS, 16 * nS, cudaMemcpyDeviceToDevice,
                       h->st));
    CK(cudaMemcpyAsync(h->out.p, (const double2*)h->rout.p + (size_t)last * nT, 16 * nT, cudaMemcpyDeviceToDevice,
                       h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  int flag = 0;
  CK(cudaMemcpy(&flag, h->dp.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag == 3) return h->fail(DEFMM_ERR_CUDA, "a tensor-core kernel's wait for its MMAs timed out");
  if (flag) return h->fail(DEFMM_ERR_ARG, "inconsistent interaction list detected on the device");
  h->has_out = true;
  return 0;
}

int defmm_gemv(defmm_handle* h, const double* in, double* out) { return defmm_gemv_batched(h, 1, in, out); }

int defmm_check_full(defmm_handle* h, int64_t nsamples, uint64_t seed, double err[3]) {
  if (!h || !err || nsamples < 1) return DEFMM_ERR_ARG;
  if (!h->built || !h->has_out) return h->fail(DEFMM_ERR_ARG, "check before a host gemv");
  CK(cudaSetDevice(h->device));
  const int64_t nS = (int64_t)h->plan.S.perm.size(), nT = (int64_t)h->plan.T.perm.size();
  nsamples = std::min(nsamples, nT);
  // seeded partial Fisher-Yates over target indices
  std::vector<int64_t> idx(nT);
  for (int64_t i = 0; i < nT; i++) idx[i] = i;
  uint64_t s = seed;
  for (int64_t i = 0; i < nsamples; i++) {
    int64_t j = i + (int64_t)(splitmix(s) % (uint64_t)(nT - i));
    std::swap(idx[i], idx[j]);
  }
  idx.resize(nsamples);
  std::sort(idx.begin(), idx.end());
  std::vector<double> tpos(3 * nsamples);
  for (int64_t i = 0; i < nsamples; i++)
    for (int k = 0; k < 3; k++) tpos[3 * i + k] = h->trg[3 * idx[i] + k];
  int st = ensure(h, h->chk, (size_t)nsamples * 40);
  if (st) return st;
  double* d_tpos = (double*)h->chk.p;
  double2* d_res = (double2*)((char*)h->chk.p + 24 * nsamples);
  CK(cudaMemcpy(d_tpos, tpos.data(), 24 * nsamples, cudaMemcpyHostToDevice));
  dfb::launch_direct(nS, h->dp.S_pos, h->dp.S_perm, (const double2*)h->qin.p, nsamples, d_tpos, h->plan.kappa,
                     d_res, h->st);
  CK(cudaGetLastError());
  std::vector<double> ex(2 * nsamples), fm(2 * nT);
  CK(cudaMemcpyAsync(ex.data(), d_res, 16 * nsamples, cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(fm.data(), h->out.p, 16 * nT, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  // gaia_vectors.hpp:119-172 norms
  double ainf = 0, binf = 0, a1 = 0, b1 = 0, a2 = 0, b2 = 0;
  for (int64_t i = 0; i < nsamples; i++) {
    const double er = ex[2 * i] - fm[2 * idx[i]], ei = ex[2 * i + 1] - fm[2 * idx[i] + 1];
    const double d = std::hypot(er, ei), m = std::hypot(ex[2 * i], ex[2 * i + 1]);
    ainf = std::max(ainf, d);
    binf = std::max(binf, m);
    a1 += d;
    b1 += m;
    a2 += d * d;
    b2 += m * m;
  }
  err[0] = ainf / binf;
  err[1] = a1 / b1;
  err[2] = std::sqrt(a2 / b2);
  return 0;
}

int defmm_info(const defmm_handle* h, int what, int64_t* v) {
  if (!h || !v) return DEFMM_ERR_ARG;
  const Plan& p = h->plan;
  switch (what) {
    case DEFMM_INFO_N_SOURCES: *v = (int64_t)h->src.size() / 3; return 0;
    case DEFMM_INFO_N_TARGETS: *v = (int64_t)h->trg.size() / 3; return 0;
    default: break;
  }
  if (!h->built) return DEFMM_ERR_ARG;
  switch (what) {
    case DEFMM_INFO_NLVL: *v = p.lv.nlvl; break;
    case DEFMM_INFO_CPT: *v = p.lv.cpt; break;
    case DEFMM_INFO_MAX_STAGE: *v = p.lv.max_stage; break;
    case DEFMM_INFO_CELLS_T: *v = p.T.ncell; break;
    case DEFMM_INFO_CELLS_S: *v = p.S.ncell; break;
    case DEFMM_INFO_SLOTS_S: *v = p.sS.n; break;
    case DEFMM_INFO_SLOTS_T: *v = p.sT.n; break;
    case DEFMM_INFO_FAR_HF: *v = p.n_far_hf; break;
    case DEFMM_INFO_FAR_LF: *v = p.n_far_lf; break;
    case DEFMM_INFO_NEAR: *v = p.n_near; break;
    case DEFMM_INFO_I_NEAR: *v = p.i_near; break;
    case DEFMM_INFO_TABLES: *v = (int64_t)p.tab_lvl.size(); break;
    case DEFMM_INFO_DEVICE_BYTES:
      *v = (int64_t)(h->dev_bytes + layout_bytes(h) + h->sig.bytes + h->sig2.bytes + h->ptab.bytes +
                     h->pnear.bytes + h->pfar.bytes + h->qin.bytes + h->out.bytes + h->rin.bytes + h->rout.bytes);
      break;
    case DEFMM_INFO_LAYOUT: *v = h->layout; break;
    case DEFMM_INFO_RHS_BLOCK: *v = h->layout == 2 ? h->gl.R : 0; break;
    case DEFMM_INFO_GROUPS: *v = h->layout == 2 ? (int64_t)h->gl.groups.size() : 0; break;
    case DEFMM_INFO_TENSOR_CORES: *v = tc_on(h) ? 1 : 0; break;
    case DEFMM_INFO_TREE_DEVICE: *v = p.tree_on_device ? 1 : 0; break;
    case DEFMM_INFO_RHS_PER_CTA: {  // the block the M2L launcher uses for the grouped layout's R
      const int R = h->layout == 2 ? h->gl.R : 1;
      int rb = std::min(h->rhs_block_m2l, h->ops ? h->ops->max_rb : 1);
      while (rb > 1 && R % rb) rb >>= 1;
      *v = rb;
      break;
    }
    case DEFMM_INFO_M2L_STAGING: *v = h->m2l_staging ? 1 : 0; break;
    case DEFMM_INFO_M2L_GROUP_LIST: *v = h->m2l_lgroup; break;
    case DEFMM_INFO_TREE_MS: *v = (int64_t)(1e3 * p.t_tree); break;
    case DEFMM_INFO_LIST_RECORDS: *v = p.keep_lists ? 1 : 0; break;
    case DEFMM_INFO_LAUNCHES: *v = h->launches; break;
    case DEFMM_INFO_PERMUTED_SPECTRA: *v = (int64_t)p.ptab_key.size(); break;
    case DEFMM_INFO_PLAN_WALK_DEVICE: *v = h->walked_on_device ? 1 : 0; break;
    case DEFMM_INFO_PLAN_MS: *v = (int64_t)(1e3 * (p.t_tree + p.t_lists + p.t_tables)); break;
    case DEFMM_INFO_PLAN_WALK_MS: *v = (int64_t)(1e3 * p.t_walk); break;
    case DEFMM_INFO_M2L_THREADS: {
      const int pi = h->precision == DEFMM_PRECISION_FP64 ? 0 : 1;
      *v = h->m2l_nt[pi] ? h->m2l_nt[pi] : (p.PP > 1024 ? 256 : 128);
      break;
    }
    case DEFMM_INFO_P2P_BLOCKS_PER_SM: *v = h->p2p_bps[h->precision == DEFMM_PRECISION_FP64 ? 0 : 1]; break;
    case DEFMM_INFO_M2L_PAIRING: *v = h->m2l_pair[h->precision == DEFMM_PRECISION_FP64 ? 0 : 1]; break;
    case DEFMM_INFO_M2L_TARGETS: {
      int64_t n = 0;
      for (int64_t k = 0; k < p.sT.n; k++) n += p.m2l_ptr[k + 1] > p.m2l_ptr[k] ? 1 : 0;
      *v = n;
      break;
    }
    case DEFMM_INFO_LEAF_SLOTS_S: {
      int64_t n = 0;
      for (int32_t c : p.p2m_leaf) n += p.sS.cell_ptr[c + 1] - p.sS.cell_ptr[c];
      *v = n;
      break;
    }
    case DEFMM_INFO_M2M_ENTRIES: *v = p.m2m_ptr.empty() ? p.n_m2m : p.m2m_ptr.back(); break;
    case DEFMM_INFO_L2L_ENTRIES: *v = p.l2l_ptr.empty() ? p.n_l2l : p.l2l_ptr.back(); break;
    case DEFMM_INFO_P2M_POINT_SLOTS: {
      int64_t n = 0;
      for (int32_t c : p.p2m_leaf) n += (int64_t)p.S.nprt[c] * (p.sS.cell_ptr[c + 1] - p.sS.cell_ptr[c]);
      *v = n;
      break;
    }
    case DEFMM_INFO_L2P_POINT_SLOTS: {
      int64_t n = 0;
      for (int32_t c : p.l2p_leaf) n += (int64_t)p.T.nprt[c] * (p.sT.cell_ptr[c + 1] - p.sT.cell_ptr[c]);
      *v = n;
      break;
    }
    case DEFMM_INFO_M2F_SLOTS: {  // source slots at precomputed levels that have target slots in their cone
      int64_t n = 0;
      for (int l = 0; l < p.lv.nlvl; l++) {
        const auto& cS = p.sS.cone_begin[l];
        const auto& cT = p.sT.cone_begin[l];
        for (size_t c = 0; c + 1 < cS.size() && c + 1 < cT.size(); c++)
          if (cT[c + 1] > cT[c]) n += cS[c + 1] - cS[c];
      }
      *v = n;
      break;
    }
    default: return DEFMM_ERR_ARG;
  }
  return 0;
}

int defmm_phase_times(const defmm_handle* h, double ms[10]) {
  if (!h || !ms) return DEFMM_ERR_ARG;
  for (int i = 0; i < PH_N; i++) ms[i] = h->phase_ms[i];
  return 0;
}

int defmm_dump_tree(const defmm_handle* h, int which, int32_t* ci, double* cd, int32_t* dirs, int64_t* ndirs,
                    int32_t* perm) {
  if (!h || !h->built || (which != 0 && which != 1)) return DEFMM_ERR_ARG;
  const dfb::Tree& t = which ? h->plan.S : h->plan.T;
  const dfb::Slots& s = which ? h->plan.sS : h->plan.sT;
  int64_t nd = 0;
  for (int64_t c = 0; c < t.ncell; c++) {
    if (ci) {
      int32_t* r = ci + 8 * c;
      r[0] = t.idx[3 * c];
      r[1] = t.idx[3 * c + 1];
      r[2] = t.idx[3 * c + 2];
      r[3] = t.lvl[c];
      r[4] = t.nprt[c];
      r[5] = t.first[c];
      r[6] = t.nson[c];
      r[7] = (int32_t)(s.cell_ptr[c + 1] - s.cell_ptr[c]);
    }
    if (cd) {
      cd[4 * c] = t.ctr[3 * c];
      cd[4 * c + 1] = t.ctr[3 * c + 1];
      cd[4 * c + 2] = t.ctr[3 * c + 2];
      cd[4 * c + 3] = t.rad[c];
    }
    for (int64_t j = s.cell_ptr[c]; j < s.cell_ptr[c + 1]; j++)
      if (s.cell_dirs[j] >= 0) {
        if (dirs) dirs[nd] = s.cell_dirs[j];
        nd++;
      }
  }
  if (ndirs) *ndirs = nd;
  if (perm) std::memcpy(perm, t.perm.data(), t.perm.size() * 4);
  return 0;
}

int defmm_dump_lists(const defmm_handle* h, int32_t* far_hf, int32_t* far_lf, int32_t* near_, int64_t n[3]) {
  if (!h || !h->built || !n) return DEFMM_ERR_ARG;
  const Plan& p = h->plan;
  n[0] = (int64_t)p.rec_far_hf.size() / 6;
  n[1] = (int64_t)p.rec_far_lf.size() / 5;
  n[2] = (int64_t)p.rec_near.size() / 2;
  if (far_hf) std::memcpy(far_hf, p.rec_far_hf.data(), p.rec_far_hf.size() * 4);
  if (far_lf) std::memcpy(far_lf, p.rec_far_lf.data(), p.rec_far_lf.size() * 4);
  if (near_) std::memcpy(near_, p.rec_near.data(), p.rec_near.size() * 4);
  return 0;
}

int defmm_dump_m2l(const defmm_handle* h, int64_t* ptr, int32_t* src, uint32_t* tab, int64_t n[2]) {
  if (!h || !h->built || !n) return DEFMM_ERR_ARG;
  const Plan& p = h->plan;
  n[0] = (int64_t)p.m2l_ptr.size();
  n[1] = p.m2l_ptr.empty() ? 0 : p.m2l_ptr.back();
  if (ptr) std::memcpy(ptr, p.m2l_ptr.data(), p.m2l_ptr.size() * 8);
  if (!src && !tab) return 0;
  if (p.dev_m2l_src) {  // entries left on the device by the level walk
    if (h->device >= 0 && cudaSetDevice(h->device) != cudaSuccess) return DEFMM_ERR_CUDA;
    if ((src && cudaMemcpy(src, p.dev_m2l_src, (size_t)n[1] * 4, cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (tab && cudaMemcpy(tab, p.dev_m2l_tab, (size_t)n[1] * 4, cudaMemcpyDeviceToHost) != cudaSuccess)) {
      cudaGetLastError();
      return DEFMM_ERR_CUDA;
    }
  } else {
    if (src) std::memcpy(src, p.m2l_src.data(), p.m2l_src.size() * 4);
    if (tab) std::memcpy(tab, p.m2l_tab.data(), p.m2l_tab.size() * 4);
  }
  if (tab)  // ids -> (table << 6) | hash keys
    for (int64_t i = 0; i < n[1]; i++) tab[i] = p.ptab_key[tab[i]];
  return 0;
}

int defmm_near_digest(const defmm_handle* h, uint64_t* digest) {
  if (!h || !h->built || !digest) return DEFMM_ERR_ARG;
  const Plan& p = h->plan;
  const Plan::NearOnDevice& d = p.nd;
  if (d.on && h->device >= 0 && cudaSetDevice(h->device) != cudaSuccess) return DEFMM_ERR_CUDA;
  int k = 0;
  bool ok = true;
  // FNV-1a over the element count and the bytes of one array, wherever it lives
  auto hash = [&](const void* host, const void* dev, int64_t n, size_t es) {
    std::vector<unsigned char> buf;
    const unsigned char* b = static_cast<const unsigned char*>(host);
    if (d.on) {
      buf.resize((size_t)n * es);
      if (n && cudaMemcpy(buf.data(), dev, (size_t)n * es, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        ok = false;
      }
      b = buf.data();
    }
    uint64_t x = 1469598103934665603ull;
    for (int s = 0; s < 64; s += 8) x = (x ^ (((uint64_t)n >> s) & 0xff)) * 1099511628211ull;
    for (size_t i = 0; i < (size_t)n * es; i++) x = (x ^ b[i]) * 1099511628211ull;
    digest[k++] = x;
  };
  auto at = [&](const std::vector<int64_t>& v, const int64_t* dv, int64_t i) -> int64_t {
    if (!d.on) return v.empty() ? 0 : v[i];
    int64_t x = 0;
    if (dv && cudaMemcpy(&x, dv + i, 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaGetLastError();
      ok = false;
    }
    return x;
  };
#define NEAR_ARRAY(vec, dptr, n) hash((vec).data(), (dptr), d.on ? (int64_t)(n) : (int64_t)(vec).size(), sizeof((vec)[0]))
  const bool sym = p.p2p_sym;
  const int64_t nch = p.near_chunks(), nit = p.near_items(), nsy = sym ? p.near_sym_items() : 0;
  const int64_t nred = sym ? p.near_red_leaves() : 0;
  const int64_t npc = at(p.p2p_ptr, d.p2p_ptr, nit);
  NEAR_ARRAY(p.p2p_tfirst, d.tfirst, nch);
  NEAR_ARRAY(p.p2p_tn, d.tn, nch);
  NEAR_ARRAY(p.p2p_ptr, d.p2p_ptr, nit + 1);
  NEAR_ARRAY(p.p2p_sfirst, d.p2p_sfirst, npc);
  NEAR_ARRAY(p.p2p_sn, d.p2p_sn, npc);
  NEAR_ARRAY(p.p2p_item_chunk, d.p2p_item_chunk, nit);
  NEAR_ARRAY(p.p2p_chunk_items, d.p2p_chunk_items, nch + 1);
  NEAR_ARRAY(p.p2p_order, d.p2p_order, nit);
  const int64_t nself = sym ? at(p.self_ptr, d.self_ptr, nch) : 0;
  const int64_t nys = sym ? at(p.sym_ptr, d.sym_ptr, nsy) : 0;
  const int64_t nro = sym ? at(p.red_ptr, d.red_ptr, nred) : 0;
  NEAR_ARRAY(p.self_ptr, d.self_ptr, sym ? nch + 1 : 0);
  NEAR_ARRAY(p.self_sfirst, d.self_sfirst, nself);
  NEAR_ARRAY(p.self_sn, d.self_sn, nself);
  NEAR_ARRAY(p.self_order, d.self_order, sym ? p.near_self_items() : 0);
  NEAR_ARRAY(p.sym_ptr, d.sym_ptr, sym ? nsy + 1 : 0);
  NEAR_ARRAY(p.sym_sfirst, d.sym_sfirst, nys);
  NEAR_ARRAY(p.sym_sn, d.sym_sn, nys);
  NEAR_ARRAY(p.sym_soff, d.sym_soff, nys);
  NEAR_ARRAY(p.sym_item_chunk, d.sym_item_chunk, nsy);
  NEAR_ARRAY(p.sym_chunk_items, d.sym_chunk_items, sym ? nch + 1 : 0);
  NEAR_ARRAY(p.sym_order, d.sym_order, nsy);
  NEAR_ARRAY(p.red_first, d.red_first, nred);
  NEAR_ARRAY(p.red_n, d.red_n, nred);
  NEAR_ARRAY(p.red_ptr, d.red_ptr, sym ? nred + 1 : 0);
  NEAR_ARRAY(p.red_off, d.red_off, nro);
#undef NEAR_ARRAY
  digest[k++] = (uint64_t)p.sym_scratch;
  digest[k++] = (uint64_t)p.i_near;
  digest[k++] = (uint64_t)p.n_near;
  return ok ? 0 : DEFMM_ERR_CUDA;
}

}  // extern "C"

int dfb::handle_view(defmm_handle* h, dfb::HandleView* v) {
  if (!h || !v) return DEFMM_ERR_ARG;
  if (!h->built || !h->has_out || !h->qin.p) return h->fail(DEFMM_ERR_ARG, "direct sums need a host gemv first");
  v->device = h->device;
  v->stream = h->st;
  v->nS = (int64_t)h->plan.S.perm.size();
  v->S_pos = h->dp.S_pos;
  v->S_perm = h->dp.S_perm;
  v->qin = (const double2*)h->qin.p;
  v->qin_read = h->ev_qin_read;
  v->kappa = h->plan.kappa;
  return 0;
}

int dfb::handle_fail(defmm_handle* h, int code, const char* msg) { return h->fail(code, msg); }
