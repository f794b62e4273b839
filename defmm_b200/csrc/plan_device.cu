// The level walk of the plan (LevelWalk: dual traversal, cones, effective
// directions, slots, far entries) on the GPU, level by level.  Same results
// as the host walk in plan.cpp, bit for bit: every floating-point decision
// (admissibility hrzpass.hpp:52-56, the cone of a translation
// newdirections.hpp:175-185) uses the host's IEEE operations in the host's
// order with explicit round-to-nearest intrinsics (no contraction), every
// list keeps the reference's depth-first order (stable compaction by prefix
// sums), and the cone of a translation comes from its first pair in that
// order (M2L.hpp:189-197).
#include <cub/cub.cuh>

#include <algorithm>
#include <memory>
#include <cstring>

#include "fp64_math.hpp"
#include "plan.hpp"
#include "plan_device.hpp"

namespace dfb {
namespace {

__constant__ int8_t c_axis_order[8][3] = {{0, 1, 2}, {1, 0, 2}, {0, 1, 2}, {1, 2, 0},
                                          {0, 2, 1}, {0, 1, 2}, {2, 0, 1}, {2, 1, 0}};

struct DTree {
  const int32_t* idx;  // 3 per cell
  const double* ctr;   // 3 per cell
  const double* rad;
  const int64_t* son_ptr;
  const int32_t* sons;
  const int32_t* parent;
  const int32_t* loc;  // level-local index
};

// sqrt((0 + x x) + y y) + z z), as the host's norm3 without contraction
__device__ __forceinline__ double dnorm3(double x, double y, double z) {
  double t = __dadd_rn(0.0, __dmul_rn(x, x));
  t = __dadd_rn(t, __dmul_rn(y, y));
  t = __dadd_rn(t, __dmul_rn(z, z));
  return __dsqrt_rn(t);
}

// 0 far, 1 near, 2 split (with the children count)
__global__ void k_classify(int64_t nf, const int2* __restrict__ F, DTree T, DTree S, int prec, int hf, double kappa,
                           int32_t* __restrict__ isfar, int32_t* __restrict__ isnear, int64_t* __restrict__ nch) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const int t = F[i].x, s = F[i].y;
  bool far = false;
  if (prec) {
    if (hf) {  // MACgeomhf
      const double dx = __dsub_rn(T.ctr[3 * t], S.ctr[3 * s]), dy = __dsub_rn(T.ctr[3 * t + 1], S.ctr[3 * s + 1]),
                   dz = __dsub_rn(T.ctr[3 * t + 2], S.ctr[3 * s + 2]);
      const double tt = __dmul_rn(2., S.rad[s]);
      const double tmp = __dmul_rn(1. - 1.e-8, __dsub_rn(dnorm3(dx, dy, dz), tt));
      const double a = __dmul_rn(__dmul_rn(tt, tt), kappa);
      const double mx = (a < tt) ? tt : a;
      far = tmp >= mx;
    } else {  // MAClist
      int test = 0, ncmp = 3;
      for (int k = 0; k < 3; k++) {
        const int d = T.idx[3 * t + k] - S.idx[3 * s + k];
        ncmp -= d ? 0 : 1;
        test += d < 0 ? -d : d;
      }
      far = test > ncmp;
    }
  }
  const int64_t nt = T.son_ptr[t + 1] - T.son_ptr[t], ns = S.son_ptr[s + 1] - S.son_ptr[s];
  const bool near = !far && (nt == 0 || ns == 0);
  isfar[i] = far ? 1 : 0;
  isnear[i] = near ? 1 : 0;
  nch[i] = (!far && !near) ? nt * ns : 0;
}

__global__ void k_scatter(int64_t nf, const int2* __restrict__ F, DTree T, DTree S, const int32_t* __restrict__ isfar,
                          const int32_t* __restrict__ pfar, const int32_t* __restrict__ isnear,
                          const int32_t* __restrict__ pnear, const int64_t* __restrict__ nch,
                          const int64_t* __restrict__ pch, int2* __restrict__ far_out, int2* __restrict__ near_out,
                          int2* __restrict__ next) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const int2 pr = F[i];
  if (isfar[i]) {
    far_out[pfar[i]] = pr;
  } else if (isnear[i]) {
    near_out[pnear[i]] = pr;
  } else if (nch[i]) {
    const int64_t ta = T.son_ptr[pr.x], tb = T.son_ptr[pr.x + 1], sa = S.son_ptr[pr.y], sb = S.son_ptr[pr.y + 1];
    int64_t o = pch[i];
    for (int64_t a = ta; a < tb; a++)
      for (int64_t b = sa; b < sb; b++) next[o++] = make_int2(T.sons[a], S.sons[b]);
  }
}

__device__ __forceinline__ void diz(const DTree& T, const DTree& S, int2 pr, int* iZ) {
  for (int k = 0; k < 3; k++) iZ[k] = T.idx[3 * pr.x + k] - S.idx[3 * pr.y + k];
}

__global__ void k_maxdiff(int64_t nf, const int2* __restrict__ P, DTree T, DTree S, int* __restrict__ m) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int v = 0;
  if (i < nf) {
    int iZ[3];
    diz(T, S, P[i], iZ);
    for (int k = 0; k < 3; k++) v = max(v, iZ[k] < 0 ? -iZ[k] : iZ[k]);
  }
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v) atomicMax(m, v);
}

__device__ __forceinline__ int64_t zkey(const DTree& T, const DTree& S, int2 pr, int m) {
  int iZ[3];
  diz(T, S, pr, iZ);
  const int64_t w = 2 * m + 1;
  return ((int64_t)(iZ[0] + m) * w + (iZ[1] + m)) * w + (iZ[2] + m);
}

__global__ void k_firstpos(int64_t nf, const int2* __restrict__ P, DTree T, DTree S, int m,
                           unsigned long long* __restrict__ first) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  atomicMin(first + zkey(T, S, P[i], m), (unsigned long long)i);
}

// the cone of each translation: direction nearest to the normalised centre
// difference of its first pair, lowest index on ties (one block per key)
__global__ void k_cones(int64_t nkeys, const unsigned long long* __restrict__ first, const int2* __restrict__ P,
                        DTree T, DTree S, const double* __restrict__ dirs, int nd, int16_t* __restrict__ key_cone) {
  __shared__ double bd[256];
  __shared__ int bi[256];
  for (int64_t k = blockIdx.x; k < nkeys; k += gridDim.x) {
    const unsigned long long f = first[k];
    if (f == ~0ULL) continue;  // uniform over the block
    const int2 pr = P[f];
    double u[3];
    for (int q = 0; q < 3; q++) u[q] = __dsub_rn(T.ctr[3 * pr.x + q], S.ctr[3 * pr.y + q]);
    const double n = dnorm3(u[0], u[1], u[2]);
    for (int q = 0; q < 3; q++) u[q] = __ddiv_rn(u[q], n);
    double best = 1.e30;
    int ind = -1;
    for (int i = threadIdx.x; i < nd; i += blockDim.x) {  // increasing i: strict < keeps the lowest
      const double d = dnorm3(__dsub_rn(dirs[3 * i], u[0]), __dsub_rn(dirs[3 * i + 1], u[1]),
                              __dsub_rn(dirs[3 * i + 2], u[2]));
      if (d < best) {
        best = d;
        ind = i;
      }
    }
    bd[threadIdx.x] = best;
    bi[threadIdx.x] = ind;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
      if ((int)threadIdx.x < o) {
        const double d2 = bd[threadIdx.x + o];
        const int i2 = bi[threadIdx.x + o];
        if (i2 >= 0 && (d2 < bd[threadIdx.x] || (d2 == bd[threadIdx.x] && (bi[threadIdx.x] < 0 || i2 < bi[threadIdx.x])))) {
          bd[threadIdx.x] = d2;
          bi[threadIdx.x] = i2;
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) key_cone[k] = (int16_t)bi[0];
    __syncthreads();
  }
}

__global__ void k_cone_of(int64_t nf, const int2* __restrict__ P, DTree T, DTree S, int m,
                          const int16_t* __restrict__ key_cone, int16_t* __restrict__ cone) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  cone[i] = key_cone[zkey(T, S, P[i], m)];
}

__global__ void k_flags(int64_t nf, const int2* __restrict__ P, DTree T, DTree S, const int16_t* __restrict__ cone,
                        int nd, uint8_t* __restrict__ effT, uint8_t* __restrict__ effS) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const int c = cone[i];
  effT[(int64_t)T.loc[P[i].x] * nd + c] = 1;
  effS[(int64_t)S.loc[P[i].y] * nd + c] = 1;
}

// child flag dt set when any of the parent's 4 dt..4 dt + 3 is (dwnpass.hpp:81-109)
__global__ void k_propagate(int64_t nc, const int32_t* __restrict__ cells, DTree Tr, int nd, int pnd,
                            const uint8_t* __restrict__ prev, uint8_t* __restrict__ eff) {
  const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= nc * nd) return;
  const int64_t i = w / nd;
  const int dt = (int)(w % nd);
  const int par = Tr.parent[cells[i]];
  const uint8_t* pe = prev + (int64_t)Tr.loc[par] * pnd + 4 * dt;
  if (pe[0] | pe[1] | pe[2] | pe[3]) eff[w] = 1;
}

// d-major copy of the flags for the cone-major slot numbering
__global__ void k_transpose(int64_t nc, int nd, const uint8_t* __restrict__ eff, int32_t* __restrict__ fl) {
  const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= nc * nd) return;
  const int64_t d = w / nc, c = w % nc;
  fl[w] = eff[c * nd + d];
}

__global__ void k_cone_starts(int nd, int64_t nc, const int32_t* __restrict__ pos, int32_t* __restrict__ out) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < nd) out[d] = pos[(int64_t)d * nc];
}

__global__ void k_slots_hf(int64_t nc, int nd, const uint8_t* __restrict__ eff, const int32_t* __restrict__ pos,
                           const int32_t* __restrict__ cells, int64_t base, int32_t* __restrict__ dense,
                           int32_t* __restrict__ scell, int32_t* __restrict__ sdir) {
  const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= nc * nd) return;
  const int64_t c = w / nd;
  const int d = (int)(w % nd);
  if (!eff[w]) {
    dense[w] = -1;
    return;
  }
  const int64_t r = pos[(int64_t)d * nc + c];
  dense[w] = (int32_t)(base + r);
  scell[r] = cells[c];
  sdir[r] = d;
}

// M2M children of the source slots of one level (upwpass.hpp:49-60, the
// host's m2m lists): parent slot r (cell pc, direction d) meets each son of
// pc holding the slot of direction d / 4 (parent at an HF stage > 0) or its
// LF slot (otherwise), in son order.  cdense maps the child level's (cell,
// direction) to its slot (HF: loc * ndc + d; LF: loc), -1 where none.
// out == nullptr: count into cnt; else write from off[r].
__global__ void k_m2m_list(int64_t np, const int32_t* __restrict__ pcell, const int32_t* __restrict__ pdir, DTree S,
                           int stage_pos, int chf, int ndc, const int32_t* __restrict__ cdense,
                           int64_t* __restrict__ cnt, const int64_t* __restrict__ off, int32_t* __restrict__ out) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= np) return;
  const int pc = pcell[r];
  const int d = pdir ? pdir[r] : -1;
  const int cd = stage_pos ? d / 4 : -1;
  int n = 0;
  const int64_t o = out ? off[r] : 0;
  for (int64_t a = S.son_ptr[pc]; a < S.son_ptr[pc + 1]; a++) {
    const int64_t loc = S.loc[S.sons[a]];
    int32_t cs = -1;
    if (chf) {
      if (cd >= 0) cs = cdense[loc * ndc + cd];
    } else if (cd < 0) {
      cs = cdense[loc];
    }
    if (cs >= 0) {
      if (out) out[o + n] = cs;
      n++;
    }
  }
  if (!out) cnt[r] = n;
}

// L2L parents of the target slots of one level (dwnpass.hpp:49-58, the
// host's l2l lists): child slot r (cell c, direction dt) meets the slots of
// its parent with directions 4 dt .. 4 dt + 3 (parent at an HF stage > 0),
// all of its slots (HF stage 0), or its LF slot, in direction order.
__global__ void k_l2l_list(int64_t nc, const int32_t* __restrict__ ccell, const int32_t* __restrict__ cdir, DTree T,
                           int stage_pos, int phf, int ndp, const int32_t* __restrict__ pdense,
                           int64_t* __restrict__ cnt, const int64_t* __restrict__ off, int32_t* __restrict__ out) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nc) return;
  const int pc = T.parent[ccell[r]];
  const int dt = cdir ? cdir[r] : -1;
  int n = 0;
  const int64_t o = out ? off[r] : 0;
  if (pc >= 0) {
    const int64_t loc = T.loc[pc];
    auto emit = [&](int32_t ps) {
      if (ps >= 0) {
        if (out) out[o + n] = ps;
        n++;
      }
    };
    if (stage_pos) {
      for (int j = 0; j < 4; j++) {
        const int d = 4 * dt + j;
        if (d >= 0 && d < ndp) emit(pdense[loc * ndp + d]);
      }
    } else if (phf) {
      for (int j = 0; j < ndp; j++) emit(pdense[loc * ndp + j]);
    } else {
      emit(pdense[loc]);
    }
  }
  if (!out) cnt[r] = n;
}

__global__ void k_tabflags(int64_t nf, const int2* __restrict__ P, DTree T, DTree S, int m, int32_t* __restrict__ used) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  int iZ[3];
  diz(T, S, P[i], iZ);
  const int a0 = abs(iZ[0]), a1 = abs(iZ[1]), a2 = abs(iZ[2]);
  const int h1 = (a0 < a1 ? 1 : 0) | (a0 < a2 ? 2 : 0) | (a1 < a2 ? 4 : 0);
  int nI[3];
  for (int k = 0; k < 3; k++) nI[k] = abs(iZ[c_axis_order[h1][k]]);
  used[((int64_t)nI[0] * (m + 1) + nI[1]) * (m + 1) + nI[2]] = 1;
}

__global__ void k_entries(int64_t nf, const int2* __restrict__ P, DTree T, DTree S, int m, int hf, int nd,
                          const int16_t* __restrict__ cone, const int32_t* __restrict__ denseT,
                          const int32_t* __restrict__ denseS, const int32_t* __restrict__ tidpos, int64_t tbase,
                          int32_t* __restrict__ ts, int32_t* __restrict__ ss, uint32_t* __restrict__ tab) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const int2 pr = P[i];
  int iZ[3];
  diz(T, S, pr, iZ);
  const int a0 = abs(iZ[0]), a1 = abs(iZ[1]), a2 = abs(iZ[2]);
  const int h1 = (a0 < a1 ? 1 : 0) | (a0 < a2 ? 2 : 0) | (a1 < a2 ? 4 : 0);
  const int h0 = (iZ[0] < 0 ? 1 : 0) | (iZ[1] < 0 ? 2 : 0) | (iZ[2] < 0 ? 4 : 0);
  int nI[3];
  for (int k = 0; k < 3; k++) nI[k] = abs(iZ[c_axis_order[h1][k]]);
  const int64_t fi = ((int64_t)nI[0] * (m + 1) + nI[1]) * (m + 1) + nI[2];
  const int64_t lt = T.loc[pr.x], ls = S.loc[pr.y];
  ts[i] = hf ? denseT[lt * nd + cone[i]] : denseT[lt];
  ss[i] = hf ? denseS[ls * nd + cone[i]] : denseS[ls];
  tab[i] = ((uint32_t)(tbase + tidpos[fi]) << 6) | (uint32_t)(h0 + (h1 << 3));
}

__global__ void k_iota(int64_t n, int32_t* __restrict__ v) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) v[i] = (int32_t)i;
}

__global__ void k_count(int64_t n, const int32_t* __restrict__ key, int32_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(cnt + key[i], 1);
}

// entries in sorted order; marks the (table, hash) keys that occur
__global__ void k_gather_entries(int64_t n, const int32_t* __restrict__ order, const int32_t* __restrict__ ss,
                                 const uint32_t* __restrict__ tab, int32_t* __restrict__ src,
                                 uint32_t* __restrict__ key, int32_t* __restrict__ used) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t o = order[i];
  src[i] = ss[o];
  key[i] = tab[o];
  used[tab[o]] = 1;
}

__global__ void k_gather_i32(int64_t n, const int32_t* __restrict__ order, const int32_t* __restrict__ in,
                             int32_t* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[order[i]];
}

__global__ void k_renumber(int64_t n, const int32_t* __restrict__ pid, uint32_t* __restrict__ key) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) key[i] = (uint32_t)pid[key[i]];
}

inline unsigned nblk(int64_t n, int b = 256) { return (unsigned)std::max<int64_t>(1, (n + b - 1) / b); }

// Device buffers of one walk; everything is freed at the end.
struct Arena {
  std::vector<void*> all;
  ~Arena() {
    for (void* p : all) cudaFree(p);
  }
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)) != cudaSuccess) return nullptr;
    all.push_back(p);
    return static_cast<T*>(p);
  }
  void drop(void* p) {
    auto it = std::find(all.begin(), all.end(), p);
    if (it != all.end()) {
      cudaFree(p);
      all.erase(it);
    }
  }
};

// One level's slots on the device during the walk: slot r has cell cell[r]
// and direction dir[r] (dir == nullptr: LF, -1); dense maps (level-local
// cell, direction) -> slot (HF: loc * nd + d; LF: loc), -1 where none.
struct LvlSlots {
  int64_t n = 0;
  const int32_t* cell = nullptr;
  const int32_t* dir = nullptr;
  const int32_t* dense = nullptr;
  int nd = 0;
  bool prec = false, hf = false, stage_pos = false;  // stage_pos: HF with HF stage > 0
  std::vector<void*> own;                            // device buffers to free with the level
};

struct DeviceWalker final : LevelWalker {
  int walk(Plan& p, LevelWalk& w, std::string& err) override;
};

#define DW_CK(call)                                                          \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      err = std::string("device plan: ") + #call + ": " + cudaGetErrorString(e_); \
      return -4;                                                             \
    }                                                                        \
  } while (0)
#define DW_ALLOC(ptr, T, n)                                      \
  do {                                                           \
    ptr = A.get<T>(n);                                           \
    if (!ptr) {                                                  \
      cudaGetLastError();                                        \
      err = "device plan: out of device memory";                 \
      return -5;                                                 \
    }                                                            \
  } while (0)

template <typename T>
int upload_vec(Arena& A, const std::vector<T>& v, const T** out, std::string& err) {
  T* p = nullptr;
  DW_ALLOC(p, T, v.size());
  if (!v.empty()) DW_CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = p;
  return 0;
}

int DeviceWalker::walk(Plan& p, LevelWalk& walk, std::string& err) {
  const Levels& v = p.lv;
  const int nlvl = v.nlvl;
  Arena A;
  // cells per level (DFS order) and level-local indices, as the host walk
  std::vector<std::vector<int32_t>> lcT(nlvl), lcS(nlvl);
  std::vector<int32_t> locT(p.T.ncell), locS(p.S.ncell);
  for (int64_t c = 0; c < p.T.ncell; c++) {
    locT[c] = (int32_t)lcT[p.T.lvl[c]].size();
    lcT[p.T.lvl[c]].push_back((int32_t)c);
  }
  for (int64_t c = 0; c < p.S.ncell; c++) {
    locS[c] = (int32_t)lcS[p.S.lvl[c]].size();
    lcS[p.S.lvl[c]].push_back((int32_t)c);
  }
  auto dtree = [&](const Tree& tr, const std::vector<int32_t>& loc, DTree& d) -> int {
    int st;
    if ((st = upload_vec(A, tr.idx, &d.idx, err)) || (st = upload_vec(A, tr.ctr, &d.ctr, err)) ||
        (st = upload_vec(A, tr.rad, &d.rad, err)) || (st = upload_vec(A, tr.son_ptr, &d.son_ptr, err)) ||
        (st = upload_vec(A, tr.sons, &d.sons, err)) || (st = upload_vec(A, tr.parent, &d.parent, err)) ||
        (st = upload_vec(A, loc, &d.loc, err)))
      return st;
    return 0;
  };
  double tstep = wall_seconds();
  DTree T{}, S{};
  int st;
  if ((st = dtree(p.T, locT, T)) || (st = dtree(p.S, locS, S))) return st;
  p.step("walk: cells per level, trees to the device", tstep);

  p.sT = Slots();
  p.sS = Slots();
  p.sT.lvl_begin.assign(nlvl + 1, 0);
  p.sS.lvl_begin.assign(nlvl + 1, 0);
  p.sT.cone_begin.assign(nlvl, {});
  p.sS.cone_begin.assign(nlvl, {});
  walk.far_ts.assign(nlvl, {});
  walk.far_ss.assign(nlvl, {});
  walk.far_tab.assign(nlvl, {});
  walk.near_pairs.clear();
  walk.tab_nI.clear();

  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  auto scan = [&](auto* in, auto* out, int64_t n) -> int {
    size_t need = 0;
    DW_CK(cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, n));
    if (need > tmp_bytes) {
      if (tmp) A.drop(tmp);
      tmp = A.get<char>(need);
      if (!tmp) {
        err = "device plan: out of device memory";
        return -5;
      }
      tmp_bytes = need;
    }
    DW_CK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, n));
    return 0;
  };
  auto last = [&](const auto* arr, int64_t i, auto& out) -> int {
    DW_CK(cudaMemcpy(&out, arr + i, sizeof(out), cudaMemcpyDeviceToHost));
    return 0;
  };

  // directions of all stages, one device table
  std::vector<int64_t> dir_off(p.dirs.size() + 1, 0);
  std::vector<double> alld;
  for (size_t e = 0; e < p.dirs.size(); e++) {
    dir_off[e] = (int64_t)(alld.size() / 3);
    alld.insert(alld.end(), p.dirs[e].begin(), p.dirs[e].end());
  }
  const double* d_dirs = nullptr;
  if ((st = upload_vec(A, alld, &d_dirs, err))) return st;

  // near pairs per level, kept on the device for the near-field lists
  std::vector<std::pair<int2*, int64_t>> lv_near;
  // each level's slots (cell, direction; no direction array: LF, -1) on the
  // device, copied to the host slot arrays once all levels are known
  struct SlotSeg {
    Slots* sl;
    int64_t off, n;
    const int32_t* cell;
    const int32_t* dir;
  };
  std::vector<SlotSeg> slot_segs;
  int64_t table_count = 0;
  // every level's slots stay on the device until the M2M / L2L transfer
  // lists are built after the walk
  std::vector<LvlSlots> lvS(nlvl), lvT(nlvl);
  double t_transfers = 0;  // wall time of the transfer lists
  double t_cells = 0;      // wall time of the per-cell slot lists
  double t_sub[4] = {0, 0, 0, 0};  // per sub-step of the level loop
  auto release_lvl = [&](LvlSlots& x) {
    for (void* q : x.own)
      if (q) A.drop(q);
    x = LvlSlots();
  };
  std::vector<int32_t*> lv_ts, lv_ss;  // far entries per level, on the device
  std::vector<uint32_t*> lv_tab;
  std::vector<int64_t> lv_n;
  std::vector<int> lv_level;
  int2* F = nullptr;
  DW_ALLOC(F, int2, 1);
  const int2 root = make_int2(0, 0);
  DW_CK(cudaMemcpy(F, &root, sizeof(int2), cudaMemcpyHostToDevice));
  int64_t nfr = 1;
  uint8_t *prevT = nullptr, *prevS = nullptr;  // flags of the previous level
  for (int l = 0; l < nlvl; l++) {
    const bool prec = v.prec[l], hf = l > 0 && v.isHF[l];
    double tsub = wall_seconds();
    auto sub = [&](int k) {  // accumulate the wall time of sub-step k of the level
      cudaDeviceSynchronize();
      const double t = wall_seconds();
      t_sub[k] += t - tsub;
      tsub = t;
    };
    // 1. classify and compact: far pairs, near pairs, next frontier
    int32_t *isfar, *isnear, *pfar, *pnear;
    int64_t *nch, *pch;
    DW_ALLOC(isfar, int32_t, nfr + 1);
    DW_ALLOC(isnear, int32_t, nfr + 1);
    DW_ALLOC(pfar, int32_t, nfr + 1);
    DW_ALLOC(pnear, int32_t, nfr + 1);
    DW_ALLOC(nch, int64_t, nfr + 1);
    DW_ALLOC(pch, int64_t, nfr + 1);
    if (nfr) k_classify<<<nblk(nfr), 256>>>(nfr, F, T, S, prec ? 1 : 0, hf ? 1 : 0, p.kappa, isfar, isnear, nch);
    DW_CK(cudaGetLastError());
    DW_CK(cudaMemset(isfar + nfr, 0, sizeof(int32_t)));
    DW_CK(cudaMemset(isnear + nfr, 0, sizeof(int32_t)));
    DW_CK(cudaMemset(nch + nfr, 0, sizeof(int64_t)));
    if ((st = scan(isfar, pfar, nfr + 1)) || (st = scan(isnear, pnear, nfr + 1)) || (st = scan(nch, pch, nfr + 1)))
      return st;
    int32_t nf = 0, nn = 0;
    int64_t nx = 0;
    if ((st = last(pfar, nfr, nf)) || (st = last(pnear, nfr, nn)) || (st = last(pch, nfr, nx))) return st;
    int2 *fp, *np_, *next;
    DW_ALLOC(fp, int2, nf);
    DW_ALLOC(np_, int2, nn);
    DW_ALLOC(next, int2, nx);
    if (nfr)
      k_scatter<<<nblk(nfr), 256>>>(nfr, F, T, S, isfar, pfar, isnear, pnear, nch, pch, fp, np_, next);
    DW_CK(cudaGetLastError());
    if (nn)
      lv_near.push_back({np_, nn});
    else
      A.drop(np_);
    for (void* q : {(void*)isfar, (void*)isnear, (void*)pfar, (void*)pnear, (void*)nch, (void*)pch, (void*)F})
      A.drop(q);
    F = next;
    nfr = nx;
    if (hf) p.n_far_hf += nf; else p.n_far_lf += nf;

    sub(0);
    // 2. fundamental index bound and (HF) the cone of each far pair
    int m = 0;
    int16_t* cone = nullptr;
    const int nd = v.nDir[l];
    if (nf) {
      int* dm;
      DW_ALLOC(dm, int, 1);
      DW_CK(cudaMemset(dm, 0, sizeof(int)));
      k_maxdiff<<<nblk(nf), 256>>>(nf, fp, T, S, dm);
      DW_CK(cudaGetLastError());
      DW_CK(cudaMemcpy(&m, dm, sizeof(int), cudaMemcpyDeviceToHost));
      A.drop(dm);
    }
    if (hf && nf) {
      const int64_t wk = 2 * (int64_t)m + 1, nk = wk * wk * wk;
      unsigned long long* first;
      int16_t* kc;
      DW_ALLOC(first, unsigned long long, nk);
      DW_ALLOC(kc, int16_t, nk);
      DW_ALLOC(cone, int16_t, nf);
      DW_CK(cudaMemset(first, 0xff, nk * sizeof(unsigned long long)));
      k_firstpos<<<nblk(nf), 256>>>(nf, fp, T, S, m, first);
      const int h = v.HFStage[l];
      k_cones<<<(unsigned)std::min<int64_t>(nk, 65535), 256>>>(nk, first, fp, T, S, d_dirs + 3 * dir_off[h],
                                                              (int)(p.dirs[h].size() / 3), kc);
      k_cone_of<<<nblk(nf), 256>>>(nf, fp, T, S, m, kc, cone);
      DW_CK(cudaGetLastError());
      A.drop(first);
      A.drop(kc);
    }

    sub(1);
    // 3. effective directions of this level (+ propagation from the parent level)
    const bool hfprec = v.prec[l] && v.isHF[l];
    const int64_t ncT = (int64_t)lcT[l].size(), ncS = (int64_t)lcS[l].size();
    uint8_t *effT = nullptr, *effS = nullptr;
    const int32_t *cellsT = nullptr, *cellsS = nullptr;
    if ((st = upload_vec(A, lcT[l], &cellsT, err)) || (st = upload_vec(A, lcS[l], &cellsS, err))) return st;
    if (hfprec) {
      DW_ALLOC(effT, uint8_t, ncT * nd);
      DW_ALLOC(effS, uint8_t, ncS * nd);
      DW_CK(cudaMemset(effT, 0, std::max<int64_t>(1, ncT * nd)));
      DW_CK(cudaMemset(effS, 0, std::max<int64_t>(1, ncS * nd)));
      if (hf && nf) k_flags<<<nblk(nf), 256>>>(nf, fp, T, S, cone, nd, effT, effS);
      if (!v.noHF && l > 0 && v.isHF[l - 1] && v.prec[l - 1] && prevT && prevS) {
        const int pnd = v.nDir[l - 1];
        if (ncT) k_propagate<<<nblk(ncT * nd), 256>>>(ncT, cellsT, T, nd, pnd, prevT, effT);
        if (ncS) k_propagate<<<nblk(ncS * nd), 256>>>(ncS, cellsS, S, nd, pnd, prevS, effS);
      }
      DW_CK(cudaGetLastError());
    }

    // 4. slots of this level (cone-major, cells in DFS order)
    int32_t *denseT = nullptr, *denseS = nullptr;
    LvlSlots curT, curS;  // this level's slots on the device (kept for the transfer lists)
    auto slots = [&](Slots& sl, const std::vector<int32_t>& cells, const int32_t* dcells, int64_t nc,
                     const uint8_t* eff, int32_t*& dense, LvlSlots& cur) -> int {
      cur.prec = v.prec[l];
      cur.hf = v.isHF[l];
      cur.stage_pos = v.isHF[l] && v.HFStage[l] > 0;
      cur.nd = nd;
      sl.lvl_begin[l] = sl.n;
      if (!v.prec[l]) {
        sl.cone_begin[l].assign(2, sl.n);
        return 0;
      }
      if (!v.isHF[l]) {  // one LF expansion per cell
        sl.cone_begin[l] = {sl.n, sl.n + nc};
        std::vector<int32_t> dh(nc);
        for (int64_t i = 0; i < nc; i++) dh[i] = (int32_t)(sl.n + i);
        slot_segs.push_back({&sl, sl.n, nc, dcells, nullptr});  // cells in slot order, direction -1
        const int32_t* dd = nullptr;
        int s2 = upload_vec(A, dh, &dd, err);
        if (s2) return s2;
        dense = const_cast<int32_t*>(dd);
        cur.n = nc;
        cur.cell = dcells;  // the level's cell list, in slot order
        cur.dir = nullptr;  // -1
        sl.n += nc;
        return 0;
      }
      int32_t *fl, *pos, *scell, *sdir;
      const int64_t tot = nc * nd;
      DW_ALLOC(fl, int32_t, tot + 1);
      DW_ALLOC(pos, int32_t, tot + 1);
      DW_ALLOC(dense, int32_t, tot);
      if (tot) k_transpose<<<nblk(tot), 256>>>(nc, nd, eff, fl);
      DW_CK(cudaMemset(fl + tot, 0, sizeof(int32_t)));
      int s2 = scan(fl, pos, tot + 1);
      if (s2) return s2;
      int32_t cnt = 0;
      if ((s2 = last(pos, tot, cnt))) return s2;
      DW_ALLOC(scell, int32_t, cnt);
      DW_ALLOC(sdir, int32_t, cnt);
      if (tot) k_slots_hf<<<nblk(tot), 256>>>(nc, nd, eff, pos, dcells, sl.n, dense, scell, sdir);
      DW_CK(cudaGetLastError());
      // cone starts: pos at (d, 0), gathered on the device (nd values of the
      // nc x nd positions)
      int32_t* cs;
      DW_ALLOC(cs, int32_t, nd);
      k_cone_starts<<<nblk(nd), 256>>>(nd, nc, pos, cs);
      DW_CK(cudaGetLastError());
      std::vector<int32_t> ph(nd);
      DW_CK(cudaMemcpy(ph.data(), cs, (size_t)nd * sizeof(int32_t), cudaMemcpyDeviceToHost));
      A.drop(cs);
      sl.cone_begin[l].assign(nd + 1, 0);
      for (int d = 0; d < nd; d++) sl.cone_begin[l][d] = sl.n + ph[d];
      sl.cone_begin[l][nd] = sl.n + cnt;
      slot_segs.push_back({&sl, sl.n, (int64_t)cnt, scell, sdir});
      A.drop(fl);
      A.drop(pos);
      cur.n = cnt;
      cur.cell = scell;
      cur.dir = sdir;
      cur.own = {scell, sdir};
      sl.n += cnt;
      return 0;
    };
    if ((st = slots(p.sT, lcT[l], cellsT, ncT, effT, denseT, curT)) ||
        (st = slots(p.sS, lcS[l], cellsS, ncS, effS, denseS, curS)))
      return st;
    curT.dense = denseT;
    curS.dense = denseS;

    sub(2);
    // 5. transfer-spectrum ids per fundamental index and the far entries
    if (nf) {
      const int64_t nkey = (int64_t)(m + 1) * (m + 1) * (m + 1);
      int32_t *used, *tpos, *ts, *ss;
      uint32_t* tab;
      DW_ALLOC(used, int32_t, nkey + 1);
      DW_ALLOC(tpos, int32_t, nkey + 1);
      DW_CK(cudaMemset(used, 0, (nkey + 1) * sizeof(int32_t)));
      k_tabflags<<<nblk(nf), 256>>>(nf, fp, T, S, m, used);
      DW_CK(cudaGetLastError());
      if ((st = scan(used, tpos, nkey + 1))) return st;
      std::vector<int32_t> uh(nkey);
      DW_CK(cudaMemcpy(uh.data(), used, nkey * sizeof(int32_t), cudaMemcpyDeviceToHost));
      const int64_t tbase = table_count;
      for (int64_t k = 0; k < nkey; k++)
        if (uh[k]) {
          table_count++;
          const int a = (int)(k / ((m + 1) * (m + 1))), b = (int)((k / (m + 1)) % (m + 1)), c = (int)(k % (m + 1));
          walk.tab_nI.push_back({a, b, c});
          p.tab_lvl.push_back(l);
          const int M = v.nCellMax[l];
          p.tab_iz.push_back(((int64_t)a * M + b) * M + c);
        }
      DW_ALLOC(ts, int32_t, nf);
      DW_ALLOC(ss, int32_t, nf);
      DW_ALLOC(tab, uint32_t, nf);
      k_entries<<<nblk(nf), 256>>>(nf, fp, T, S, m, hf ? 1 : 0, nd, cone, denseT, denseS, tpos, tbase, ts, ss, tab);
      DW_CK(cudaGetLastError());
      lv_ts.push_back(ts);  // kept on the device for the M2L grouping below
      lv_ss.push_back(ss);
      lv_tab.push_back(tab);
      lv_n.push_back(nf);
      lv_level.push_back(l);
      for (void* q : {(void*)used, (void*)tpos}) A.drop(q);
    }
    if (cone) A.drop(cone);
    A.drop(fp);
    sub(3);
    // this level's slots, dense maps and cell lists: kept for the transfer lists
    curS.own.push_back(denseS);
    curS.own.push_back(const_cast<int32_t*>(cellsS));
    curT.own.push_back(denseT);
    curT.own.push_back(const_cast<int32_t*>(cellsT));
    lvS[l] = curS;
    lvT[l] = curT;
    if (prevT) A.drop(prevT);
    if (prevS) A.drop(prevS);
    prevT = effT;
    prevS = effS;
  }
  {  // the slots' cells and directions to the host: arrays sized once, one copy per level
    const double tc = wall_seconds();
    for (Slots* sl : {&p.sT, &p.sS}) {
      sl->cell.resize(sl->n);
      sl->dir.resize(sl->n);
    }
    for (const SlotSeg& g : slot_segs) {
      if (g.n == 0) continue;
      DW_CK(cudaMemcpy(g.sl->cell.data() + g.off, g.cell, (size_t)g.n * sizeof(int32_t), cudaMemcpyDeviceToHost));
      if (g.dir)
        DW_CK(cudaMemcpy(g.sl->dir.data() + g.off, g.dir, (size_t)g.n * sizeof(int32_t), cudaMemcpyDeviceToHost));
      else
        std::fill(g.sl->dir.begin() + g.off, g.sl->dir.begin() + g.off + g.n, -1);
    }
    t_sub[2] += wall_seconds() - tc;
  }
  // per-cell slot lists (each cell's slots in slot order, so its directions
  // increase): a stable radix sort of all slots by cell.  The slots' cells
  // and directions and the per-cell slot ids and directions stay on the
  // device; the pointers and directions also go to the host (cell_slots
  // stays empty there)
  if (p.sT.n < ((int64_t)1 << 31) - 1 && p.sS.n < ((int64_t)1 << 31) - 1) {
    const double tc = wall_seconds();
    auto csr = [&](Slots& sl, const Tree& tr, void** dcell, void** ddirs, void** dslot, void** ddir) -> int {
      const int64_t n = sl.n, nc = tr.ncell;
      int32_t *idx, *keys, *cnt;
      int64_t* ptr;
      DW_ALLOC(idx, int32_t, n);
      DW_ALLOC(keys, int32_t, n);
      DW_ALLOC(cnt, int32_t, nc + 1);
      DW_ALLOC(ptr, int64_t, nc + 1);
      for (void** q : {dcell, ddirs, dslot, ddir})
        if (cudaMalloc(q, std::max<int64_t>(1, n) * sizeof(int32_t)) != cudaSuccess) {  // handed to the plan's owner
          cudaGetLastError();
          *q = nullptr;
          err = "device plan: out of device memory";
          return -5;
        }
      int32_t* cell = static_cast<int32_t*>(*dcell);  // per slot: cell, direction
      int32_t* dir = static_cast<int32_t*>(*ddirs);
      int32_t* cslot = static_cast<int32_t*>(*dslot);  // per cell: slots, directions
      int32_t* cdir = static_cast<int32_t*>(*ddir);
      for (const SlotSeg& g : slot_segs) {
        if (g.sl != &sl || g.n == 0) continue;
        DW_CK(cudaMemcpy(cell + g.off, g.cell, (size_t)g.n * sizeof(int32_t), cudaMemcpyDeviceToDevice));
        if (g.dir)
          DW_CK(cudaMemcpy(dir + g.off, g.dir, (size_t)g.n * sizeof(int32_t), cudaMemcpyDeviceToDevice));
        else
          DW_CK(cudaMemset(dir + g.off, 0xff, (size_t)g.n * sizeof(int32_t)));  // -1
      }
      DW_CK(cudaMemset(cnt, 0, (nc + 1) * sizeof(int32_t)));
      if (n) {
        k_iota<<<nblk(n), 256>>>(n, idx);
        k_count<<<nblk(n), 256>>>(n, cell, cnt);
        int bits = 1;
        while (bits < 31 && ((int64_t)1 << bits) <= nc) bits++;
        size_t need = 0;
        DW_CK(cub::DeviceRadixSort::SortPairs(nullptr, need, cell, keys, idx, cslot, (int)n, 0, bits));
        char* t2 = A.get<char>(need);
        if (!t2) {
          err = "device plan: out of device memory";
          return -5;
        }
        DW_CK(cub::DeviceRadixSort::SortPairs(t2, need, cell, keys, idx, cslot, (int)n, 0, bits));
        A.drop(t2);
        k_gather_i32<<<nblk(n), 256>>>(n, cslot, dir, cdir);
        DW_CK(cudaGetLastError());
      }
      int st2 = scan(cnt, ptr, nc + 1);
      if (st2) return st2;
      sl.cell_ptr.resize(nc + 1);
      sl.cell_dirs.resize(n);
      sl.cell_slots.clear();
      DW_CK(cudaMemcpy(sl.cell_ptr.data(), ptr, (nc + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
      DW_CK(cudaMemcpy(sl.cell_dirs.data(), cdir, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost));
      for (void* q : {(void*)idx, (void*)keys, (void*)cnt, (void*)ptr}) A.drop(q);
      return 0;
    };
    if ((st = csr(p.sT, p.T, &p.dev_scell_T, &p.dev_sdir_T, &p.dev_cslot_T, &p.dev_cdir_T)) ||
        (st = csr(p.sS, p.S, &p.dev_scell_S, &p.dev_sdir_S, &p.dev_cslot_S, &p.dev_cdir_S)))
      return st;
    walk.cells_done = true;
    t_cells = wall_seconds() - tc;
  }
  // M2M lists of every source slot (children: the next level) and L2L lists
  // of every target slot (parents: the previous level), counted per level
  // into one array over all slots, one scan, then filled; left on the device
  const double t_tr = wall_seconds();
  auto transfers = [&](const Slots& sl, const std::vector<LvlSlots>& lv, const DTree& tr, bool m2m,
                       void** ptr_out, void** ent_out, int64_t* n_out) -> int {
    const int64_t n = sl.n;
    int64_t* cnt;  // 64-bit, so that the scan's sums cannot overflow
    DW_ALLOC(cnt, int64_t, n + 1);
    DW_CK(cudaMemset(cnt, 0, (n + 1) * sizeof(int64_t)));
    int64_t* ptr = nullptr;
    if (cudaMalloc(&ptr, (n + 1) * sizeof(int64_t)) != cudaSuccess) {
      cudaGetLastError();
      err = "device plan: out of device memory";
      return -5;
    }
    *ptr_out = ptr;  // handed to the plan's owner (also on error: freed there)
    for (int pass = 0; pass < 2; pass++) {
      if (pass == 1) {
        int s2 = scan(cnt, ptr, n + 1);
        if (s2) return s2;
        if ((s2 = last(ptr, n, *n_out))) return s2;
        if (cudaMalloc(ent_out, std::max<int64_t>(1, *n_out) * sizeof(int32_t)) != cudaSuccess) {
          cudaGetLastError();
          err = "device plan: out of device memory";
          return -5;
        }
      }
      for (int l = 0; l < nlvl; l++) {
        const LvlSlots& a = lv[l];  // the slots whose lists are built
        const int lb = m2m ? l + 1 : l - 1;
        if (a.n == 0 || lb < 0 || lb >= nlvl) continue;
        const LvlSlots& b = lv[lb];
        if (!b.dense || !b.prec || b.n == 0) continue;
        const int64_t base = sl.lvl_begin[l];
        int32_t* out = pass ? static_cast<int32_t*>(*ent_out) : nullptr;
        const int64_t* off = pass ? ptr + base : nullptr;
        if (m2m)
          k_m2m_list<<<nblk(a.n), 256>>>(a.n, a.cell, a.dir, tr, a.stage_pos ? 1 : 0, b.hf ? 1 : 0, b.nd, b.dense,
                                         cnt + base, off, out);
        else
          k_l2l_list<<<nblk(a.n), 256>>>(a.n, a.cell, a.dir, tr, b.stage_pos ? 1 : 0, b.hf ? 1 : 0, b.nd, b.dense,
                                         cnt + base, off, out);
        DW_CK(cudaGetLastError());
      }
    }
    A.drop(cnt);
    return 0;
  };
  if ((st = transfers(p.sS, lvS, S, true, &p.dev_m2m_ptr, &p.dev_m2m_child, &p.n_m2m)) ||
      (st = transfers(p.sT, lvT, T, false, &p.dev_l2l_ptr, &p.dev_l2l_parent, &p.n_l2l)))
    return st;
  for (int l = 0; l < nlvl; l++) {
    release_lvl(lvS[l]);
    release_lvl(lvT[l]);
  }
  p.m2m_ptr.clear();
  p.m2m_child.clear();
  p.l2l_ptr.clear();
  p.l2l_parent.clear();
  t_transfers = wall_seconds() - t_tr;
  walk.transfers_done = true;
  p.sT.lvl_begin[nlvl] = p.sT.n;
  p.sS.lvl_begin[nlvl] = p.sS.n;
  p.step("walk: levels, other (allocations, copies)", tstep);
  p.t_steps.back().second -= t_transfers + t_cells + t_sub[0] + t_sub[1] + t_sub[2] + t_sub[3];
  p.t_steps.push_back({"walk: levels, pair classification and near pairs", t_sub[0]});
  p.t_steps.push_back({"walk: levels, cones of the far pairs", t_sub[1]});
  p.t_steps.push_back({"walk: levels, effective directions and slots", t_sub[2]});
  p.t_steps.push_back({"walk: levels, far entries", t_sub[3]});
  p.t_steps.push_back({"walk: M2M and L2L transfer lists", t_transfers});
  if (walk.cells_done) p.t_steps.push_back({"walk: slots per cell (radix sort by cell)", t_cells});

  // the near-field work lists from all levels' near pairs (walk order),
  // built and kept on the device
  {
    double tn0 = wall_seconds();
    int64_t nn = 0;
    for (auto& x : lv_near) nn += x.second;
    int2* all_near;
    DW_ALLOC(all_near, int2, nn);
    int64_t o = 0;
    for (auto& x : lv_near) {
      DW_CK(cudaMemcpy(all_near + o, x.first, x.second * sizeof(int2), cudaMemcpyDeviceToDevice));
      A.drop(x.first);
      o += x.second;
    }
    lv_near.clear();
    p.n_near = nn;
    st = device_near_lists(p, all_near, nn, err);
    if (st == -5) {  // beyond device memory or 32-bit sort sizes: the host builds the lists
      std::vector<int2> near_h((size_t)nn);
      DW_CK(cudaMemcpy(near_h.data(), all_near, (size_t)nn * sizeof(int2), cudaMemcpyDeviceToHost));
      walk.near_pairs.resize(near_h.size());
      for (size_t i = 0; i < near_h.size(); i++) walk.near_pairs[i] = {near_h[i].x, near_h[i].y};
      p.nd = Plan::NearOnDevice();
      p.i_near = 0;
      p.sym_scratch = 0;
      err.clear();
      st = 0;
    } else if (st) {
      return st;
    } else {
      walk.near_done = true;
    }
    A.drop(all_near);
    p.step("walk: near-field lists (ranges, chunks, symmetric blocks, work items)", tn0);
  }

  // M2L entries grouped by target slot: a stable radix sort of all levels'
  // entries (level order, then walk order) by target slot, as the host's
  // counting placement; then the permuted-spectrum ids (one per
  // (table, hash) key that occurs, in increasing key order)
  int64_t n = 0;
  for (int64_t c : lv_n) n += c;
  if (n >= ((int64_t)1 << 31) - 1) {  // beyond 32-bit sort indices: the host groups the entries
    for (size_t q = 0; q < lv_n.size(); q++) {
      const int l = lv_level[q];
      walk.far_ts[l].resize(lv_n[q]);
      walk.far_ss[l].resize(lv_n[q]);
      walk.far_tab[l].resize(lv_n[q]);
      DW_CK(cudaMemcpy(walk.far_ts[l].data(), lv_ts[q], lv_n[q] * 4, cudaMemcpyDeviceToHost));
      DW_CK(cudaMemcpy(walk.far_ss[l].data(), lv_ss[q], lv_n[q] * 4, cudaMemcpyDeviceToHost));
      DW_CK(cudaMemcpy(walk.far_tab[l].data(), lv_tab[q], lv_n[q] * 4, cudaMemcpyDeviceToHost));
    }
    return 0;
  }
  int32_t *all_ts, *all_ss, *idx, *keys_out, *idx_out, *cnt, *used, *pid;
  uint32_t* all_tab;
  DW_ALLOC(all_ts, int32_t, n);
  DW_ALLOC(all_ss, int32_t, n);
  DW_ALLOC(all_tab, uint32_t, n);
  {
    int64_t o = 0;
    for (size_t k = 0; k < lv_n.size(); k++) {
      DW_CK(cudaMemcpy(all_ts + o, lv_ts[k], lv_n[k] * 4, cudaMemcpyDeviceToDevice));
      DW_CK(cudaMemcpy(all_ss + o, lv_ss[k], lv_n[k] * 4, cudaMemcpyDeviceToDevice));
      DW_CK(cudaMemcpy(all_tab + o, lv_tab[k], lv_n[k] * 4, cudaMemcpyDeviceToDevice));
      A.drop(lv_ts[k]);
      A.drop(lv_ss[k]);
      A.drop(lv_tab[k]);
      o += lv_n[k];
    }
  }
  DW_ALLOC(idx, int32_t, n);
  DW_ALLOC(keys_out, int32_t, n);
  DW_ALLOC(idx_out, int32_t, n);
  if (n) k_iota<<<nblk(n), 256>>>(n, idx);
  // entries grouped by target slot and, within a slot, by increasing source
  // slot: a stable sort by source, then a stable sort by target
  auto sort_by = [&](const int32_t* keys, int64_t range, int32_t* vin, int32_t* vout) -> int {
    int bits = 1;
    while (bits < 31 && ((int64_t)1 << bits) <= range) bits++;
    size_t need = 0;
    DW_CK(cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_out, vin, vout, n, 0, bits));
    char* t2 = A.get<char>(need);
    if (!t2) {
      err = "device plan: out of device memory";
      return -5;
    }
    DW_CK(cub::DeviceRadixSort::SortPairs(t2, need, keys, keys_out, vin, vout, n, 0, bits));
    A.drop(t2);
    return 0;
  };
  if ((st = sort_by(all_ss, p.sS.n, idx, idx_out))) return st;  // idx_out: entries by source
  {
    int32_t* ts_by_src = A.get<int32_t>(std::max<int64_t>(1, n));
    if (!ts_by_src) {
      err = "device plan: out of device memory";
      return -5;
    }
    if (n) k_gather_i32<<<nblk(n), 256>>>(n, idx_out, all_ts, ts_by_src);
    if ((st = sort_by(ts_by_src, p.sT.n, idx_out, idx))) return st;  // idx: by target, then source
    A.drop(ts_by_src);
    std::swap(idx, idx_out);  // the gather below reads idx_out
  }
  const int64_t nslot = p.sT.n, ntab = (int64_t)walk.tab_nI.size() * 64;
  DW_ALLOC(cnt, int32_t, nslot + 1);
  DW_ALLOC(used, int32_t, ntab + 1);
  DW_ALLOC(pid, int32_t, ntab + 1);
  DW_CK(cudaMemset(cnt, 0, (nslot + 1) * sizeof(int32_t)));
  DW_CK(cudaMemset(used, 0, (ntab + 1) * sizeof(int32_t)));
  void *src_out = nullptr, *key_out = nullptr;  // handed to the plan's owner
  DW_CK(cudaMalloc(&src_out, std::max<int64_t>(1, n) * sizeof(int32_t)));
  if (cudaMalloc(&key_out, std::max<int64_t>(1, n) * sizeof(uint32_t)) != cudaSuccess) {
    cudaFree(src_out);
    cudaGetLastError();
    err = "device plan: out of device memory";
    return -5;
  }
  auto fail_out = [&](int code) {
    cudaFree(src_out);
    cudaFree(key_out);
    return code;
  };
  if (n) {
    k_count<<<nblk(n), 256>>>(n, all_ts, cnt);
    k_gather_entries<<<nblk(n), 256>>>(n, idx_out, all_ss, all_tab, (int32_t*)src_out, (uint32_t*)key_out, used);
  }
  if (cudaGetLastError() != cudaSuccess) return fail_out(-4);
  int32_t* pos = nullptr;
  pos = A.get<int32_t>(nslot + 1);
  if (!pos) return fail_out(-5);
  if ((st = scan(cnt, pos, nslot + 1)) || (st = scan(used, pid, ntab + 1))) return fail_out(st);
  if (n) k_renumber<<<nblk(n), 256>>>(n, pid, (uint32_t*)key_out);
  const cudaError_t esync = cudaDeviceSynchronize();
  p.step("walk: far entries by target slot (radix sorts)", tstep);
  if (esync != cudaSuccess) {
    cudaGetLastError();
    err = "device plan: M2L grouping failed";
    return fail_out(-4);
  }
  std::vector<int32_t> ph(nslot + 1), uh(ntab);
  if (cudaMemcpy(ph.data(), pos, (nslot + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
      (ntab && cudaMemcpy(uh.data(), used, ntab * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)) {
    cudaGetLastError();
    err = "device plan: copy of the M2L grouping failed";
    return fail_out(-4);
  }
  p.m2l_ptr.assign(ph.begin(), ph.end());
  p.ptab_key.clear();
  for (int64_t k = 0; k < ntab; k++)
    if (uh[k]) p.ptab_key.push_back((uint32_t)k);
  p.dev_m2l_src = src_out;
  p.dev_m2l_tab = key_out;
  p.n_m2l = n;
  walk.m2l_done = true;
  p.step("walk: M2L pointers and spectrum ids to the host", tstep);
  return 0;
}

}  // namespace

// ------------------------------------------------------ octree on the device --
// The particle side of the octree build (TreeSorter): per level, each
// particle of a splitting cell gets its bit code sum_k (x_k > c_k) << k
// against the cell centre the host computed, the codes are counted per
// (cell, octant), and every particle is keyed by the first position of its
// new cell (its child's, or its own cell's when the cell stays); a stable
// radix sort by that key moves the particles of every splitting cell into
// its children's ranges in octant order, keeping their order within a child
// (sort.hpp:98-170).  cf[i] is the first position of the cell of the
// particle at position i; at[cf] maps a cell of the current level to its
// index (-1 for cells that stay).
__global__ void k_tree_mark(int64_t m, const int64_t* __restrict__ first, const uint8_t* __restrict__ split,
                            int32_t* __restrict__ at) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < m) at[first[j]] = split[j] ? (int32_t)j : -1;
}

__global__ void k_tree_codes(int64_t n, const double* __restrict__ pts, const int32_t* __restrict__ order,
                             const int32_t* __restrict__ cf, const int32_t* __restrict__ at,
                             const double* __restrict__ ctr, uint8_t* __restrict__ code, int32_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t s = at[cf[i]];
  if (s < 0) {
    code[i] = 255;
    return;
  }
  const double* x = pts + 3 * (int64_t)order[i];
  const double* c = ctr + 3 * (int64_t)s;
  const int b = (x[0] > c[0] ? 1 : 0) | (x[1] > c[1] ? 2 : 0) | (x[2] > c[2] ? 4 : 0);
  code[i] = (uint8_t)b;
  atomicAdd(&cnt[8 * s + b], 1);
}

__global__ void k_tree_keys(int64_t n, const int32_t* __restrict__ cf, const int32_t* __restrict__ at,
                            const uint8_t* __restrict__ code, const int64_t* __restrict__ child_first,
                            int32_t* __restrict__ key) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t b = code[i];
  key[i] = b == 255 ? cf[i] : (int32_t)child_first[8 * (int64_t)at[cf[i]] + b];
}

struct DeviceSorter final : TreeSorter {
  int64_t n = 0;
  int bits = 1;
  double* pts = nullptr;
  int32_t *order = nullptr, *order2 = nullptr, *cf = nullptr, *key = nullptr, *at = nullptr, *cnt = nullptr;
  uint8_t* code = nullptr;
  int64_t *first = nullptr, *childf = nullptr;
  double* ctr = nullptr;
  uint8_t* split = nullptr;
  int64_t cap = 0;  // cells per level the level arrays hold
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  cudaStream_t st = nullptr;
  void release() {
    for (void* p : {(void*)pts, (void*)order, (void*)order2, (void*)cf, (void*)key, (void*)at, (void*)cnt,
                    (void*)code, (void*)first, (void*)childf, (void*)ctr, (void*)split, tmp})
      if (p) cudaFree(p);
    pts = nullptr;
    order = order2 = cf = key = at = cnt = nullptr;
    code = nullptr;
    first = childf = nullptr;
    ctr = nullptr;
    split = nullptr;
    tmp = nullptr;
    tmp_bytes = 0;
    cap = 0;
    if (st) cudaStreamDestroy(st);
    st = nullptr;
  }
  ~DeviceSorter() override { release(); }
  int fail(std::string& err, const char* what, cudaError_t e) {
    err = std::string("device tree: ") + what + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    release();
    return e == cudaErrorMemoryAllocation ? -5 : -4;
  }
  int begin(const double* p, int64_t np, std::string& err) override {
    release();
    n = np;
    bits = 1;
    while (bits < 31 && ((int64_t)1 << bits) <= n) bits++;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&pts, 24 * (size_t)n)) != cudaSuccess ||
        (e = cudaMalloc(&order, 4 * (size_t)n)) != cudaSuccess ||
        (e = cudaMalloc(&order2, 4 * (size_t)n)) != cudaSuccess || (e = cudaMalloc(&cf, 4 * (size_t)n)) != cudaSuccess ||
        (e = cudaMalloc(&key, 4 * (size_t)n)) != cudaSuccess || (e = cudaMalloc(&at, 4 * (size_t)n)) != cudaSuccess ||
        (e = cudaMalloc(&code, (size_t)n)) != cudaSuccess)
      return fail(err, "allocation", e);
    if ((e = cudaMemcpyAsync(pts, p, 24 * (size_t)n, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(cf, 0, 4 * (size_t)n, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(at, 0xff, 4 * (size_t)n, st)) != cudaSuccess)
      return fail(err, "upload", e);
    k_iota<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, order);
    size_t need = 0;
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, need, key, cf, order, order2, (int)n, 0, bits, st)) !=
        cudaSuccess)
      return fail(err, "sort size", e);
    if ((e = cudaMalloc(&tmp, need)) != cudaSuccess) return fail(err, "allocation", e);
    tmp_bytes = need;
    return 0;
  }
  int histogram(int64_t m, const int64_t* f, const double* c, const uint8_t* sp, int64_t* hist,
                std::string& err) override {
    cudaError_t e;
    if (m > cap) {
      for (void* q : {(void*)first, (void*)childf, (void*)ctr, (void*)split, (void*)cnt})
        if (q) cudaFree(q);
      first = childf = nullptr;
      ctr = nullptr;
      split = nullptr;
      cnt = nullptr;
      cap = std::max<int64_t>(m, 1024);
      if ((e = cudaMalloc(&first, 8 * cap)) != cudaSuccess || (e = cudaMalloc(&childf, 64 * cap)) != cudaSuccess ||
          (e = cudaMalloc(&ctr, 24 * cap)) != cudaSuccess || (e = cudaMalloc(&split, cap)) != cudaSuccess ||
          (e = cudaMalloc(&cnt, 32 * cap)) != cudaSuccess)
        return fail(err, "allocation", e);
    }
    if ((e = cudaMemcpyAsync(first, f, 8 * m, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(ctr, c, 24 * m, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(split, sp, m, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(cnt, 0, 32 * m, st)) != cudaSuccess)
      return fail(err, "level upload", e);
    k_tree_mark<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(m, first, split, at);
    k_tree_codes<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, pts, order, cf, at, ctr, code, cnt);
    std::vector<int32_t> h(8 * m);
    if ((e = cudaMemcpyAsync(h.data(), cnt, 32 * m, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return fail(err, "level histogram", e);
    for (int64_t i = 0; i < 8 * m; i++) hist[i] = h[i];
    last_m = m;
    return 0;
  }
  int reorder(const int64_t* child_first, std::string& err) override {
    // the level's cells are those of the last histogram call
    cudaError_t e;
    if ((e = cudaMemcpyAsync(childf, child_first, 64 * last_m, cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return fail(err, "level upload", e);
    k_tree_keys<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, cf, at, code, childf, key);
    size_t tb = tmp_bytes;
    if ((e = cub::DeviceRadixSort::SortPairs(tmp, tb, key, cf, order, order2, (int)n, 0, bits, st)) !=
        cudaSuccess)
      return fail(err, "sort", e);
    std::swap(order, order2);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(err, "sort", e);
    return 0;
  }
  int finish(int32_t* out, std::string& err) override {
    cudaError_t e;
    if ((e = cudaMemcpyAsync(out, order, 4 * (size_t)n, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return fail(err, "download", e);
    release();
    return 0;
  }
  int64_t last_m = 0;
};

LevelWalker* device_level_walker() {
  static DeviceWalker w;
  return &w;
}

std::unique_ptr<TreeSorter> make_device_tree_sorter() { return std::unique_ptr<TreeSorter>(new DeviceSorter()); }

// ------------------------------------------ transfer spectra and signatures --
// The host plan's FP64 tables computed on the device with the same IEEE
// operations in the same order (this file is built without FMA contraction;
// sin and cos are sincos_fp64 on both sides), so they are bit-identical to
// the host's.
//
// Transfer spectrum of table k (circulant.hpp:133-144): the kernel
// exp(i kappa R) / (4 pi R) at R = |2 nI r + r tabZ_i| on the P^3 circulant
// grid (r: the level's cell radius), then the unnormalised forward 3-D DFT by
// definition, last axis first; one CTA per table, one line per thread.
constexpr int kMaxGrid = 15;  // P = 2L - 1 at the largest order (8)

__global__ void k_spectra(int64_t ntab, int P, const int32_t* __restrict__ fund, const double* __restrict__ rad,
                          const double* __restrict__ tabZ, double kappa, const double2* __restrict__ tw,
                          double2* __restrict__ out) {
  extern __shared__ double2 sx[];
  const int PP = P * P * P;
  for (int64_t k = blockIdx.x; k < ntab; k += gridDim.x) {
    const double r = rad[k];
    double v[3];
    for (int a = 0; a < 3; a++) v[a] = __dmul_rn(__dmul_rn(2., (double)fund[3 * k + a]), r);
    for (int i = threadIdx.x; i < PP; i += blockDim.x) {
      double t = 0.;
      for (int a = 0; a < 3; a++) {
        const double z = __dadd_rn(v[a], __dmul_rn(tabZ[3 * i + a], r));
        t = __dadd_rn(t, __dmul_rn(z, z));
      }
      const double R = __dsqrt_rn(t);
      double sn, cs;
      sincos_fp64(__dmul_rn(R, kappa), sn, cs);
      const double den = __dmul_rn(__dmul_rn(4., M_PI), R);
      sx[i] = make_double2(__ddiv_rn(cs, den), __ddiv_rn(sn, den));
    }
    __syncthreads();
    int inner = 1;
    for (int axis = 2; axis >= 0; axis--) {
      for (int ln = threadIdx.x; ln < P * P; ln += blockDim.x) {
        double2* b = sx + (int64_t)(ln / inner) * P * inner + ln % inner;
        double2 line[kMaxGrid], res[kMaxGrid];
        for (int j = 0; j < P; j++) line[j] = b[j * inner];
        for (int q = 0; q < P; q++) {
          double ar = 0., ai = 0.;
          for (int j = 0, m = 0; j < P; j++, m = (m + q) % P) {
            const double2 x = line[j], w = tw[m];
            ar = __dadd_rn(ar, __dsub_rn(__dmul_rn(x.x, w.x), __dmul_rn(x.y, w.y)));
            ai = __dadd_rn(ai, __dadd_rn(__dmul_rn(x.x, w.y), __dmul_rn(x.y, w.x)));
          }
          res[q] = make_double2(ar, ai);
        }
        for (int q = 0; q < P; q++) b[q * inner] = res[q];
      }
      __syncthreads();
      inner *= P;
    }
    for (int i = threadIdx.x; i < PP; i += blockDim.x) out[k * PP + i] = sx[i];
    __syncthreads();
  }
}

// Signatures of one HF stage (planewave.hpp:44-69): entry (d, k) =
// exp(-i kappa dir_d . x_k) on the stage's grid, and its square.
__global__ void k_signatures(int64_t n, int LL, const double* __restrict__ dirs, const double* __restrict__ nodes,
                             double kappa, double2* __restrict__ s1, double2* __restrict__ s2) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = e / LL;
    const int k = (int)(e - d * LL);
    double dp = 0.;
    for (int a = 0; a < 3; a++) dp = __dadd_rn(dp, __dmul_rn(dirs[3 * d + a], nodes[3 * k + a]));
    double sn, cs;
    sincos_fp64(__dmul_rn(kappa, dp), sn, cs);
    const double re = cs, im = -sn;
    s1[e] = make_double2(re, im);
    s2[e] = make_double2(__dsub_rn(__dmul_rn(re, re), __dmul_rn(im, im)),
                         __dadd_rn(__dmul_rn(re, im), __dmul_rn(im, re)));
  }
}

__global__ void k_to_float(int64_t n, const double2* __restrict__ in, float2* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = make_float2(__double2float_rn(in[i].x), __double2float_rn(in[i].y));
}

int device_plan_tables(const Plan& p, double2* tables, double2* sig, double2* sig2, std::string& err) {
  auto fail = [&](const char* what, cudaError_t e) {
    err = std::string("device tables: ") + what + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return -4;
  };
  std::vector<void*> tmp;
  auto up = [&](const void* src, size_t bytes, void** dst) -> cudaError_t {
    cudaError_t e = cudaMalloc(dst, std::max<size_t>(1, bytes));
    if (e != cudaSuccess) return e;
    tmp.push_back(*dst);
    return bytes ? cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  auto release = [&]() {
    for (void* q : tmp) cudaFree(q);
  };
  cudaError_t e = cudaSuccess;
  const int64_t ntab = (int64_t)p.tab_fund.size();
  if (ntab) {
    std::vector<int32_t> fund(3 * ntab);
    std::vector<double> rad(ntab), tw(2 * p.P);
    for (int64_t k = 0; k < ntab; k++) {
      for (int a = 0; a < 3; a++) fund[3 * k + a] = p.tab_fund[k][a];
      rad[k] = p.box_rad / (double)(1 << p.tab_lvl[k]);
    }
    dft_twiddles(p.P, tw.data());
    void *dfund, *drad, *dz, *dtw;
    if ((e = up(fund.data(), fund.size() * 4, &dfund)) != cudaSuccess ||
        (e = up(rad.data(), rad.size() * 8, &drad)) != cudaSuccess ||
        (e = up(p.tabZ.data(), p.tabZ.size() * 8, &dz)) != cudaSuccess ||
        (e = up(tw.data(), tw.size() * 8, &dtw)) != cudaSuccess) {
      release();
      return fail("upload", e);
    }
    const size_t smem = sizeof(double2) * (size_t)p.PP;
    if ((e = cudaFuncSetAttribute(k_spectra, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) {
      release();
      return fail("attribute", e);
    }
    k_spectra<<<(unsigned)std::min<int64_t>(ntab, 65535), 256, smem>>>(
        ntab, p.P, (const int32_t*)dfund, (const double*)drad, (const double*)dz, p.kappa, (const double2*)dtw, tables);
  }
  int64_t off = 0;
  for (size_t h = 0; h < p.sig.size() && h < 32; h++) {
    const int64_t n = (int64_t)p.sig[h].size();
    if (!n) continue;
    int lvl = -1;  // the level whose HF stage is h
    for (int l = 2; l < p.lv.nlvl; l++)
      if (p.lv.prec[l] && p.lv.isHF[l] && p.lv.HFStage[l] == (int)h) lvl = l;
    if (lvl < 0 || n != (int64_t)(p.dirs[h].size() / 3) * p.LL) {
      release();
      err = "device tables: signature layout";
      return -4;
    }
    const double alpha = .5 * (p.box_rad / (double)(1 << lvl));
    std::vector<double> nodes(3 * (size_t)p.LL);
    for (int k = 0; k < p.LL; k++) {
      const int I[3] = {k / (p.L * p.L), (k / p.L) % p.L, k % p.L};
      for (int a = 0; a < 3; a++) nodes[3 * k + a] = node_coord(I[a], p.L, alpha);
    }
    void *dd, *dn;
    if ((e = up(p.dirs[h].data(), p.dirs[h].size() * 8, &dd)) != cudaSuccess ||
        (e = up(nodes.data(), nodes.size() * 8, &dn)) != cudaSuccess) {
      release();
      return fail("upload", e);
    }
    k_signatures<<<(unsigned)std::min<int64_t>((n + 255) / 256, 65535), 256>>>(
        n, p.LL, (const double*)dd, (const double*)dn, p.kappa, sig + off, sig2 + off);
    off += n;
  }
  e = cudaDeviceSynchronize();
  release();
  if (e != cudaSuccess) return fail("kernels", e);
  return 0;
}

void tables_to_float(const double2* in, float2* out, int64_t n, cudaStream_t s) {
  if (n) k_to_float<<<(unsigned)std::min<int64_t>((n + 255) / 256, 65535), 256, 0, s>>>(n, in, out);
}

}  // namespace dfb
