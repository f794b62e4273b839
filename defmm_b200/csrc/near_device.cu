// The near-field work lists built on the device from the level walk's near
// pairs: source ranges per target leaf (merged where they touch), chunks of
// <= 32 targets, the symmetric decomposition (own-leaf blocks, symmetric
// blocks with their scratch rows, the rows to reduce per source leaf) and
// the work items with their execution order.  Contents and order are the
// host build's, element for element (plan.cpp: the near-field section of
// build_plan, build_symmetric_near, split_items, order_by_decreasing); the
// near field itself is P2P.hpp:43-79 applied to whole subtrees.
//
// Every step is a count pass, a CUB scan and a fill pass, or a stable CUB
// radix sort where the host groups or orders:
//   ranges per leaf   one entry per (near pair, leaf below its target),
//                     sorted by (leaf, first source, size) as the host's
//                     std::sort of each leaf's ranges;
//   merge             a range starts a new merged range unless it begins
//                     where the previous range of its leaf ends;
//   rows per leaf     one entry per (symmetric row, source leaf it covers),
//                     stable-sorted by leaf (the host's row order per leaf);
//   orders            stable sorts by decreasing work (the host's counting
//                     sort is stable too).
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "plan.hpp"
#include "plan_device.hpp"

namespace dfb {
namespace {

constexpr int kNT = 256;
constexpr int64_t kItemSources = Plan::kItemSources;

int nblk(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kNT - 1) / kNT, 1 << 16)); }
int nblk_warps(int64_t n) { return nblk(n * 32); }

#define GRID_LOOP(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_iota(int64_t n, int32_t* v) {
  GRID_LOOP(i, n) v[i] = (int32_t)i;
}

// leaf flags of the target cells (n + 1 entries, the last 0)
__global__ void k_leaf_flags(int64_t n, const int32_t* __restrict__ nson, int32_t* __restrict__ f) {
  GRID_LOOP(c, n + 1) f[c] = c < n && nson[c] == 0 ? 1 : 0;
}

__global__ void k_leaf_list(int64_t n, const int32_t* __restrict__ nson, const int32_t* __restrict__ lpre,
                            int32_t* __restrict__ leaves) {
  GRID_LOOP(c, n) if (nson[c] == 0) leaves[lpre[c]] = (int32_t)c;
}

// particle -> ordinal of its leaf (one warp per leaf)
__global__ void k_particle_leaf(int64_t nleaf, const int32_t* __restrict__ leaves, const int32_t* __restrict__ first,
                                const int32_t* __restrict__ nprt, int32_t* __restrict__ lidx) {
  const int lane = threadIdx.x & 31;
  for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < nleaf;
       w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int c = leaves[w];
    for (int k = lane; k < nprt[c]; k += 32) lidx[first[c] + k] = (int32_t)w;
  }
}

// per near pair (t, s): the leaves below t and the pair's interactions
__global__ void k_pair_count(int64_t np, const int2* __restrict__ near, const int32_t* __restrict__ sub_end,
                             const int32_t* __restrict__ lpre, const int32_t* __restrict__ tnprt,
                             const int32_t* __restrict__ snprt, int64_t* __restrict__ cnt,
                             int64_t* __restrict__ inter) {
  GRID_LOOP(i, np) {
    const int2 pr = near[i];
    cnt[i] = lpre[sub_end[pr.x]] - lpre[pr.x];
    inter[i] = (int64_t)tnprt[pr.x] * snprt[pr.y];
  }
}

// one entry per (pair, leaf below its target): key = source size, value =
// (leaf << 32) | first source
__global__ void k_pair_emit(int64_t np, const int2* __restrict__ near, const int32_t* __restrict__ lpre,
                            const int64_t* __restrict__ off, const int32_t* __restrict__ leaves,
                            const int32_t* __restrict__ sfirst, const int32_t* __restrict__ snprt,
                            uint32_t* __restrict__ key_sn, uint64_t* __restrict__ val_csf) {
  GRID_LOOP(i, np) {
    const int2 pr = near[i];
    const int64_t o = off[i], n = off[i + 1] - o;
    const int32_t l0 = lpre[pr.x];
    const uint32_t sf = (uint32_t)sfirst[pr.y], sn = (uint32_t)snprt[pr.y];
    for (int64_t m = 0; m < n; m++) {
      key_sn[o + m] = sn;
      val_csf[o + m] = ((uint64_t)(uint32_t)leaves[l0 + m] << 32) | sf;
    }
  }
}

// a sorted range opens a merged range unless it continues the previous one
// of the same leaf (E + 1 entries, the last 0)
__global__ void k_merge_head(int64_t E, const uint64_t* __restrict__ csf, const uint32_t* __restrict__ sn,
                             int32_t* __restrict__ head) {
  GRID_LOOP(k, E + 1) {
    int32_t h = 0;
    if (k == 0) {
      h = E > 0 ? 1 : 0;
    } else if (k < E) {
      const uint64_t a = csf[k - 1], b = csf[k];
      h = ((a >> 32) != (b >> 32) || (uint32_t)a + sn[k - 1] != (uint32_t)b) ? 1 : 0;
    }
    head[k] = h;
  }
}

// merged range g (gsc: exclusive scan of head): leaf, first source, end
__global__ void k_merge_fill(int64_t E, const uint64_t* __restrict__ csf, const uint32_t* __restrict__ sn,
                             const int32_t* __restrict__ head, const int64_t* __restrict__ gsc,
                             int32_t* __restrict__ mc, int32_t* __restrict__ msf, int32_t* __restrict__ mend,
                             int32_t* __restrict__ nm) {
  GRID_LOOP(k, E) {
    const int64_t g = gsc[k + 1] - 1;
    const uint64_t v = csf[k];
    if (head[k]) {
      mc[g] = (int32_t)(v >> 32);
      msf[g] = (int32_t)(uint32_t)v;
      atomicAdd(&nm[v >> 32], 1);
    }
    if (k == E - 1 || head[k + 1]) mend[g] = (int32_t)((uint32_t)v + sn[k]);
  }
}

// chunks (<= 32 targets) per leaf with ranges and their range count
__global__ void k_chunk_counts(int64_t n, const int32_t* __restrict__ nm, const int32_t* __restrict__ nprt,
                               int64_t* __restrict__ nchk, int64_t* __restrict__ nrg, int64_t* __restrict__ nm64) {
  GRID_LOOP(c, n + 1) {
    const int64_t k = c < n && nm[c] ? (nprt[c] + 31) / 32 : 0;
    nchk[c] = k;
    nrg[c] = c < n ? k * nm[c] : 0;
    nm64[c] = c < n ? nm[c] : 0;
  }
}

// one warp per leaf: its chunks and, per chunk, all the leaf's merged ranges
__global__ void k_chunk_fill(int64_t n, const int32_t* __restrict__ nm, const int64_t* __restrict__ mstart,
                             const int64_t* __restrict__ ch_off, const int64_t* __restrict__ rg_off,
                             const int32_t* __restrict__ first, const int32_t* __restrict__ nprt,
                             const int32_t* __restrict__ msf, const int32_t* __restrict__ mend,
                             int32_t* __restrict__ tfirst, int32_t* __restrict__ tn, int32_t* __restrict__ cleaf,
                             int64_t* __restrict__ ptr, int32_t* __restrict__ osf, int32_t* __restrict__ osn) {
  const int lane = threadIdx.x & 31;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n;
       c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t k = nm[c];
    if (k == 0) continue;
    const int64_t nq = ch_off[c + 1] - ch_off[c], m0 = mstart[c], r0 = rg_off[c];
    for (int64_t e = lane; e < nq * k; e += 32) {
      const int64_t j = e % k;
      osf[r0 + e] = msf[m0 + j];
      osn[r0 + e] = mend[m0 + j] - msf[m0 + j];
    }
    for (int64_t q = lane; q < nq; q += 32) {
      const int64_t ch = ch_off[c] + q;
      tfirst[ch] = first[c] + (int32_t)(32 * q);
      tn[ch] = min(32, nprt[c] - (int32_t)(32 * q));
      cleaf[ch] = (int32_t)c;
      ptr[ch + 1] = r0 + (q + 1) * k;
    }
  }
}

// symmetric decomposition per chunk: the own leaf [a0, a1) as a plain block,
// the part of each range after the own leaf as a symmetric block
__global__ void k_sym_count(int64_t nch, const int32_t* __restrict__ cleaf, const int32_t* __restrict__ first,
                            const int32_t* __restrict__ nprt, const int64_t* __restrict__ ptr,
                            const int32_t* __restrict__ sf, const int32_t* __restrict__ sn,
                            int64_t* __restrict__ nself, int64_t* __restrict__ nsym, int64_t* __restrict__ nsrc) {
  GRID_LOOP(ch, nch + 1) {
    int64_t a = 0, b = 0, s = 0;
    if (ch < nch) {
      const int32_t lf = cleaf[ch], a0 = first[lf], a1 = a0 + nprt[lf];
      for (int64_t r = ptr[ch]; r < ptr[ch + 1]; r++) {
        const int32_t s0 = sf[r], s1 = s0 + sn[r];
        if (s0 < a1 && s1 > a0) a++;
        const int32_t b0 = max(s0, a1);
        if (b0 < s1) {
          b++;
          s += s1 - b0;
        }
      }
    }
    nself[ch] = a;
    nsym[ch] = b;
    nsrc[ch] = s;
  }
}

__global__ void k_sym_fill(int64_t nch, const int32_t* __restrict__ cleaf, const int32_t* __restrict__ first,
                           const int32_t* __restrict__ nprt, const int64_t* __restrict__ ptr,
                           const int32_t* __restrict__ sf, const int32_t* __restrict__ sn,
                           const int64_t* __restrict__ self_ptr, const int64_t* __restrict__ sym_ptr,
                           const int64_t* __restrict__ src_off, int32_t* __restrict__ self_sf,
                           int32_t* __restrict__ self_sn, int32_t* __restrict__ sym_sf, int32_t* __restrict__ sym_sn,
                           int64_t* __restrict__ sym_soff, uint32_t* __restrict__ ws_key) {
  GRID_LOOP(ch, nch) {
    const int32_t lf = cleaf[ch], a0 = first[lf], a1 = a0 + nprt[lf];
    int64_t ks = self_ptr[ch], ky = sym_ptr[ch], tot = src_off[ch], ws = 0;
    for (int64_t r = ptr[ch]; r < ptr[ch + 1]; r++) {
      const int32_t s0 = sf[r], s1 = s0 + sn[r];
      if (s0 < a1 && s1 > a0) {
        self_sf[ks] = a0;
        self_sn[ks++] = a1 - a0;
        ws += a1 - a0;
      }
      const int32_t b0 = max(s0, a1);
      if (b0 < s1) {
        sym_sf[ky] = b0;
        sym_sn[ky] = s1 - b0;
        sym_soff[ky++] = tot;
        tot += s1 - b0;
      }
    }
    ws_key[ch] = ~(uint32_t)ws;  // decreasing own-leaf work
  }
}

// source leaves covered by each symmetric row (the host's walk leaf by leaf)
__global__ void k_row_count(int64_t nrow, const int32_t* __restrict__ sf, const int32_t* __restrict__ sn,
                            const int32_t* __restrict__ lidx, const int32_t* __restrict__ leaves,
                            const int32_t* __restrict__ nprt, int64_t* __restrict__ cnt) {
  GRID_LOOP(r, nrow + 1) {
    int64_t k = 0;
    if (r < nrow)
      for (int32_t j = sf[r]; j < sf[r] + sn[r]; j += nprt[leaves[lidx[j]]]) k++;
    cnt[r] = k;
  }
}

__global__ void k_row_emit(int64_t nrow, const int32_t* __restrict__ sf, const int32_t* __restrict__ sn,
                           const int64_t* __restrict__ soff, const int32_t* __restrict__ lidx,
                           const int32_t* __restrict__ leaves, const int32_t* __restrict__ nprt,
                           const int64_t* __restrict__ roff, uint32_t* __restrict__ key, int64_t* __restrict__ val,
                           int32_t* __restrict__ rc) {
  GRID_LOOP(r, nrow) {
    int64_t o = roff[r];
    for (int32_t j = sf[r]; j < sf[r] + sn[r];) {
      const int32_t lo = lidx[j];
      key[o] = (uint32_t)lo;
      val[o++] = soff[r] + (j - sf[r]);
      atomicAdd(&rc[lo], 1);
      j += nprt[leaves[lo]];
    }
  }
}

// source leaves receiving rows, in leaf order (nleaf + 1 flags, the last 0)
__global__ void k_red_flags(int64_t nleaf, const int32_t* __restrict__ rc, int32_t* __restrict__ f,
                            int64_t* __restrict__ rc64) {
  GRID_LOOP(l, nleaf + 1) {
    f[l] = l < nleaf && rc[l] > 0 ? 1 : 0;
    rc64[l] = l < nleaf ? rc[l] : 0;
  }
}

__global__ void k_red_fill(int64_t nleaf, const int32_t* __restrict__ rc, const int32_t* __restrict__ fpos,
                           const int64_t* __restrict__ rcs, const int32_t* __restrict__ leaves,
                           const int32_t* __restrict__ first, const int32_t* __restrict__ nprt,
                           int32_t* __restrict__ red_first, int32_t* __restrict__ red_n,
                           int64_t* __restrict__ red_ptr) {
  GRID_LOOP(l, nleaf) {
    if (rc[l] > 0) {
      const int32_t q = fpos[l], c = leaves[l];
      red_first[q] = first[c];
      red_n[q] = nprt[c];
      red_ptr[q + 1] = rcs[l] + rc[l];
    }
  }
}

// own-leaf work per chunk > 0 (n + 1 entries, the last 0)
__global__ void k_positive(int64_t n, const uint32_t* __restrict__ key, int32_t* __restrict__ f) {
  GRID_LOOP(i, n + 1) f[i] = i < n && key[i] != ~0u ? 1 : 0;
}

// work items: a chunk's ranges cut into items of <= kItemSources sources
__global__ void k_split_count(int64_t nch, const int64_t* __restrict__ ptr, const int32_t* __restrict__ sn,
                              int64_t* __restrict__ nit, int64_t* __restrict__ npc) {
  GRID_LOOP(ch, nch + 1) {
    int64_t fill = 0, pieces = 0, its = 0;
    if (ch < nch) {
      for (int64_t r = ptr[ch]; r < ptr[ch + 1]; r++)
        for (int32_t o = 0; o < sn[r];) {
          const int32_t take = (int32_t)min((int64_t)(sn[r] - o), kItemSources - fill);
          pieces++;
          fill += take;
          o += take;
          if (fill == kItemSources) {
            its++;
            fill = 0;
          }
        }
      if (fill) its++;
    }
    nit[ch] = its;
    npc[ch] = pieces;
  }
}

__global__ void k_split_fill(int64_t nch, const int64_t* __restrict__ ptr, const int32_t* __restrict__ sf,
                             const int32_t* __restrict__ sn, const int64_t* __restrict__ soff,
                             const int32_t* __restrict__ tn, const int64_t* __restrict__ nit,
                             const int64_t* __restrict__ npc, int64_t* __restrict__ nptr, int32_t* __restrict__ nsf,
                             int32_t* __restrict__ nsn, int64_t* __restrict__ nso, int32_t* __restrict__ chunk,
                             uint32_t* __restrict__ work_key) {
  GRID_LOOP(ch, nch) {
    int tp = 32;
    if (tn) {  // lanes per source: the chunk's targets rounded up to a power of two (>= 4)
      tp = 4;
      while (tp < tn[ch]) tp <<= 1;
    }
    int64_t fill = 0, q = npc[ch], it = nit[ch];
    for (int64_t r = ptr[ch]; r < ptr[ch + 1]; r++)
      for (int32_t o = 0; o < sn[r];) {
        const int32_t take = (int32_t)min((int64_t)(sn[r] - o), kItemSources - fill);
        nsf[q] = sf[r] + o;
        nsn[q] = take;
        if (soff) nso[q] = soff[r] + o;
        q++;
        fill += take;
        o += take;
        if (fill == kItemSources) {
          nptr[it + 1] = q;
          chunk[it] = (int32_t)ch;
          work_key[it++] = ~(uint32_t)(fill * tp);
          fill = 0;
        }
      }
    if (fill) {
      nptr[it + 1] = q;
      chunk[it] = (int32_t)ch;
      work_key[it++] = ~(uint32_t)(fill * tp);
    }
  }
}

#undef GRID_LOOP

// Device memory of one build: scratch freed at the end, outputs handed to
// the plan on success (freed here on failure).
struct Mem {
  std::vector<void*> tmp, out;
  void* cub = nullptr;
  size_t cub_bytes = 0;
  ~Mem() {
    for (void* q : tmp) cudaFree(q);
    for (void* q : out) cudaFree(q);
    if (cub) cudaFree(cub);
  }
  template <class T>
  T* get(int64_t n, bool keep = false) {
    void* q = nullptr;
    if (cudaMalloc(&q, (size_t)std::max<int64_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    (keep ? out : tmp).push_back(q);
    return static_cast<T*>(q);
  }
  void drop(void* q) {
    for (auto& x : tmp)
      if (x == q) {
        cudaFree(q);
        x = nullptr;
      }
  }
  bool temp(size_t need) {
    if (need <= cub_bytes) return true;
    if (cub) cudaFree(cub);
    cub = nullptr;
    cub_bytes = 0;
    if (cudaMalloc(&cub, need) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    cub_bytes = need;
    return true;
  }
};

}  // namespace

#define NL_CK(x)                                                         \
  do {                                                                   \
    cudaError_t e_ = (x);                                                \
    if (e_ != cudaSuccess) {                                             \
      err = std::string("device near lists: ") + cudaGetErrorString(e_); \
      return -4;                                                         \
    }                                                                    \
  } while (0)
#define NL_GET(ptr, T, n, keep)                         \
  do {                                                  \
    if (!((ptr) = M.get<T>((n), (keep)))) {             \
      err = "device near lists: out of device memory";  \
      return -5;                                        \
    }                                                   \
  } while (0)

int device_near_lists(Plan& p, const int2* d_near, int64_t npair, std::string& err) {
  const Tree &T = p.T, &S = p.S;
  Plan::NearOnDevice& o = p.nd;
  o = Plan::NearOnDevice();
  Mem M;
  const int64_t nc = T.ncell;
  auto up = [&](const std::vector<int32_t>& v, const int32_t** d) -> int {
    int32_t* q;
    NL_GET(q, int32_t, (int64_t)v.size(), false);
    NL_CK(cudaMemcpy(q, v.data(), v.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    *d = q;
    return 0;
  };
  auto scan = [&](auto* in, auto* out, int64_t n) -> int {
    size_t need = 0;
    NL_CK(cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, (int)n));
    if (!M.temp(need)) {
      err = "device near lists: out of device memory";
      return -5;
    }
    NL_CK(cub::DeviceScan::ExclusiveSum(M.cub, need, in, out, (int)n));
    return 0;
  };
  // stable sort of (key, value) pairs by key (keys in [0, 2^bits))
  auto sort = [&](auto* kin, auto* kout, auto* vin, auto* vout, int64_t n, int bits) -> int {
    size_t need = 0;
    NL_CK(cub::DeviceRadixSort::SortPairs(nullptr, need, kin, kout, vin, vout, (int)n, 0, bits));
    if (!M.temp(need)) {
      err = "device near lists: out of device memory";
      return -5;
    }
    NL_CK(cub::DeviceRadixSort::SortPairs(M.cub, need, kin, kout, vin, vout, (int)n, 0, bits));
    return 0;
  };
  auto last = [&](const auto* arr, int64_t i, auto& v) -> int {
    NL_CK(cudaMemcpy(&v, arr + i, sizeof(v), cudaMemcpyDeviceToHost));
    return 0;
  };
  auto bits_for = [](int64_t n) {
    int b = 1;
    while (b < 64 && (int64_t(1) << b) <= n) b++;
    return b;
  };
  int st;
  const int32_t *t_nson, *t_first, *t_nprt, *t_sub, *s_first, *s_nprt;
  if ((st = up(T.nson, &t_nson)) || (st = up(T.first, &t_first)) || (st = up(T.nprt, &t_nprt)) ||
      (st = up(T.sub_end, &t_sub)) || (st = up(S.first, &s_first)) || (st = up(S.nprt, &s_nprt)))
    return st;

  // target leaves in cell order, their prefix count per cell
  int32_t *lf, *lpre, *leaves;
  NL_GET(lf, int32_t, nc + 1, false);
  NL_GET(lpre, int32_t, nc + 1, false);
  k_leaf_flags<<<nblk(nc + 1), kNT>>>(nc, t_nson, lf);
  if ((st = scan(lf, lpre, nc + 1))) return st;
  int32_t nleaf = 0;
  if ((st = last(lpre, nc, nleaf))) return st;
  NL_GET(leaves, int32_t, nleaf, false);
  k_leaf_list<<<nblk(nc), kNT>>>(nc, t_nson, lpre, leaves);
  NL_CK(cudaGetLastError());

  // 1. one source range per (near pair, leaf below its target)
  int64_t *cnt, *off, *inter;
  NL_GET(cnt, int64_t, npair + 1, false);
  NL_GET(off, int64_t, npair + 1, false);
  NL_GET(inter, int64_t, npair + 1, false);
  NL_CK(cudaMemset(cnt, 0, (size_t)(npair + 1) * 8));
  NL_CK(cudaMemset(inter, 0, (size_t)(npair + 1) * 8));
  if (npair) k_pair_count<<<nblk(npair), kNT>>>(npair, d_near, t_sub, lpre, t_nprt, s_nprt, cnt, inter);
  NL_CK(cudaGetLastError());
  if ((st = scan(cnt, off, npair + 1))) return st;
  int64_t E = 0;
  if ((st = last(off, npair, E))) return st;
  {  // interactions: sum of the pairs' products
    int64_t* tot;
    NL_GET(tot, int64_t, 1, false);
    size_t need = 0;
    NL_CK(cub::DeviceReduce::Sum(nullptr, need, inter, tot, (int)(npair + 1)));
    if (!M.temp(need)) return (err = "device near lists: out of device memory", -5);
    NL_CK(cub::DeviceReduce::Sum(M.cub, need, inter, tot, (int)(npair + 1)));
    if ((st = last(tot, 0, p.i_near))) return st;
  }
  if (E >= (int64_t(1) << 31)) return (err = "device near lists: too many near-field ranges", -5);
  M.drop(cnt);
  M.drop(inter);
  uint32_t *k0, *k1;
  uint64_t *v0, *v1;
  NL_GET(k0, uint32_t, E, false);
  NL_GET(k1, uint32_t, E, false);
  NL_GET(v0, uint64_t, E, false);
  NL_GET(v1, uint64_t, E, false);
  if (npair) k_pair_emit<<<nblk(npair), kNT>>>(npair, d_near, lpre, off, leaves, s_first, s_nprt, k0, v0);
  NL_CK(cudaGetLastError());
  M.drop(off);
  // by (leaf, first, size): size first, then stably by (leaf, first)
  if (E) {
    const int bn = bits_for((int64_t)S.pos.size() / 3 + 1);
    if ((st = sort(k0, k1, v0, v1, E, bn))) return st;
    if ((st = sort(v1, v0, k1, k0, E, 32 + bits_for(nc)))) return st;
  }
  // now v0 = (leaf, first) and k0 = size, in order

  // 2. merge touching ranges per leaf
  int32_t *head, *mc, *msf, *mend, *nm;
  int64_t* gsc;
  NL_GET(head, int32_t, E + 1, false);
  NL_GET(gsc, int64_t, E + 1, false);
  k_merge_head<<<nblk(E + 1), kNT>>>(E, v0, k0, head);
  if ((st = scan(head, gsc, E + 1))) return st;
  int64_t nmg = 0;
  if ((st = last(gsc, E, nmg))) return st;
  NL_GET(mc, int32_t, nmg, false);
  NL_GET(msf, int32_t, nmg, false);
  NL_GET(mend, int32_t, nmg, false);
  NL_GET(nm, int32_t, nc + 1, false);
  NL_CK(cudaMemset(nm, 0, (size_t)(nc + 1) * 4));
  if (E) k_merge_fill<<<nblk(E), kNT>>>(E, v0, k0, head, gsc, mc, msf, mend, nm);
  NL_CK(cudaGetLastError());
  for (void* q : {(void*)k0, (void*)k1, (void*)v0, (void*)v1, (void*)head, (void*)gsc}) M.drop(q);

  // 3. chunks of <= 32 targets per leaf, each with all its leaf's ranges
  int64_t *nchk, *nrg, *nm64, *ch_off, *rg_off, *mstart;
  NL_GET(nchk, int64_t, nc + 1, false);
  NL_GET(nrg, int64_t, nc + 1, false);
  NL_GET(nm64, int64_t, nc + 1, false);
  NL_GET(ch_off, int64_t, nc + 1, false);
  NL_GET(rg_off, int64_t, nc + 1, false);
  NL_GET(mstart, int64_t, nc + 1, false);
  k_chunk_counts<<<nblk(nc + 1), kNT>>>(nc, nm, t_nprt, nchk, nrg, nm64);
  if ((st = scan(nchk, ch_off, nc + 1)) || (st = scan(nrg, rg_off, nc + 1)) || (st = scan(nm64, mstart, nc + 1)))
    return st;
  int64_t nch = 0, nrange = 0;
  if ((st = last(ch_off, nc, nch)) || (st = last(rg_off, nc, nrange))) return st;
  int32_t *tfirst, *tn, *cleaf, *rsf, *rsn;
  int64_t* rptr;
  NL_GET(tfirst, int32_t, nch, true);
  NL_GET(tn, int32_t, nch, true);
  NL_GET(cleaf, int32_t, nch, false);
  NL_GET(rptr, int64_t, nch + 1, false);
  NL_GET(rsf, int32_t, nrange, false);
  NL_GET(rsn, int32_t, nrange, false);
  NL_CK(cudaMemset(rptr, 0, 8));
  k_chunk_fill<<<nblk_warps(nc), kNT>>>(nc, nm, mstart, ch_off, rg_off, t_first, t_nprt, msf, mend, tfirst, tn, cleaf,
                                         rptr, rsf, rsn);
  NL_CK(cudaGetLastError());
  for (void* q : {(void*)nchk, (void*)nrg, (void*)nm64, (void*)ch_off, (void*)rg_off, (void*)mstart, (void*)mc,
                  (void*)msf, (void*)mend, (void*)nm})
    M.drop(q);
  o.nchunk = nch;
  o.tfirst = tfirst;
  o.tn = tn;

  // work items of a chunk CSR (ptr over chunks into sf / sn / soff): the
  // item CSR, pieces, item -> chunk, chunk -> first item, execution order
  struct Items {
    int64_t *ptr = nullptr, *chunk_items = nullptr, *soff = nullptr;
    int32_t *sf = nullptr, *sn = nullptr, *chunk = nullptr, *order = nullptr;
    int64_t n = 0;
  };
  auto split = [&](const int64_t* ptr, const int32_t* sf, const int32_t* sn, const int64_t* soff,
                   const int32_t* tn_lanes, Items& it) -> int {
    int64_t *nit, *npc;
    NL_GET(nit, int64_t, nch + 1, false);
    NL_GET(npc, int64_t, nch + 1, false);
    NL_GET(it.chunk_items, int64_t, nch + 1, true);
    int64_t* npcs;
    NL_GET(npcs, int64_t, nch + 1, false);
    k_split_count<<<nblk(nch + 1), kNT>>>(nch, ptr, sn, nit, npc);
    int s2;
    if ((s2 = scan(nit, it.chunk_items, nch + 1)) || (s2 = scan(npc, npcs, nch + 1))) return s2;
    int64_t npiece = 0;
    if ((s2 = last(it.chunk_items, nch, it.n)) || (s2 = last(npcs, nch, npiece))) return s2;
    NL_GET(it.ptr, int64_t, it.n + 1, true);
    NL_GET(it.sf, int32_t, npiece, true);
    NL_GET(it.sn, int32_t, npiece, true);
    if (soff) NL_GET(it.soff, int64_t, npiece, true);
    NL_GET(it.chunk, int32_t, it.n, true);
    NL_GET(it.order, int32_t, it.n, true);
    uint32_t *wk, *wk2;
    int32_t* idx;
    NL_GET(wk, uint32_t, it.n, false);
    NL_GET(wk2, uint32_t, it.n, false);
    NL_GET(idx, int32_t, it.n, false);
    NL_CK(cudaMemset(it.ptr, 0, 8));
    if (nch)
      k_split_fill<<<nblk(nch), kNT>>>(nch, ptr, sf, sn, soff, tn_lanes, it.chunk_items, npcs, it.ptr, it.sf, it.sn,
                                       it.soff, it.chunk, wk);
    k_iota<<<nblk(it.n), kNT>>>(it.n, idx);
    NL_CK(cudaGetLastError());
    if (it.n && (s2 = sort(wk, wk2, idx, it.order, it.n, 32))) return s2;
    for (void* q : {(void*)nit, (void*)npc, (void*)npcs, (void*)wk, (void*)wk2, (void*)idx}) M.drop(q);
    return 0;
  };

  if (p.p2p_sym) {
    // 4. own-leaf blocks and symmetric blocks per chunk
    int64_t *nself, *nsym, *nsrc, *self_ptr, *sym_cptr, *src_off;
    NL_GET(nself, int64_t, nch + 1, false);
    NL_GET(nsym, int64_t, nch + 1, false);
    NL_GET(nsrc, int64_t, nch + 1, false);
    NL_GET(self_ptr, int64_t, nch + 1, true);
    NL_GET(sym_cptr, int64_t, nch + 1, false);
    NL_GET(src_off, int64_t, nch + 1, false);
    k_sym_count<<<nblk(nch + 1), kNT>>>(nch, cleaf, t_first, t_nprt, rptr, rsf, rsn, nself, nsym, nsrc);
    if ((st = scan(nself, self_ptr, nch + 1)) || (st = scan(nsym, sym_cptr, nch + 1)) ||
        (st = scan(nsrc, src_off, nch + 1)))
      return st;
    int64_t ns = 0, nrow = 0;
    if ((st = last(self_ptr, nch, ns)) || (st = last(sym_cptr, nch, nrow)) || (st = last(src_off, nch, p.sym_scratch)))
      return st;
    int32_t *self_sf, *self_sn, *ysf, *ysn;
    int64_t* ysoff;
    uint32_t *wsk, *wsk2;
    int32_t *idx, *self_ord;
    NL_GET(self_sf, int32_t, ns, true);
    NL_GET(self_sn, int32_t, ns, true);
    NL_GET(ysf, int32_t, nrow, false);
    NL_GET(ysn, int32_t, nrow, false);
    NL_GET(ysoff, int64_t, nrow, false);
    NL_GET(wsk, uint32_t, nch + 1, false);
    NL_GET(wsk2, uint32_t, nch, false);
    NL_GET(idx, int32_t, nch, false);
    NL_GET(self_ord, int32_t, nch, true);
    if (nch)
      k_sym_fill<<<nblk(nch), kNT>>>(nch, cleaf, t_first, t_nprt, rptr, rsf, rsn, self_ptr, sym_cptr, src_off, self_sf,
                                     self_sn, ysf, ysn, ysoff, wsk);
    k_iota<<<nblk(nch), kNT>>>(nch, idx);
    NL_CK(cudaGetLastError());
    // chunks with own-leaf work, by decreasing work (stable)
    if (nch && (st = sort(wsk, wsk2, idx, self_ord, nch, 32))) return st;
    {
      int32_t *pf, *pfs;
      NL_GET(pf, int32_t, nch + 1, false);
      NL_GET(pfs, int32_t, nch + 1, false);
      k_positive<<<nblk(nch + 1), kNT>>>(nch, wsk, pf);
      if ((st = scan(pf, pfs, nch + 1))) return st;
      int32_t npos = 0;
      if ((st = last(pfs, nch, npos))) return st;
      o.n_self_order = npos;
    }
    o.self_ptr = self_ptr;
    o.self_sfirst = self_sf;
    o.self_sn = self_sn;
    o.self_order = self_ord;

    // 5. scratch rows per source leaf, in row order
    int32_t* lidx;
    NL_GET(lidx, int32_t, (int64_t)T.pos.size() / 3, false);
    k_particle_leaf<<<nblk_warps(nleaf), kNT>>>(nleaf, leaves, t_first, t_nprt, lidx);
    int64_t *rl, *roff;
    NL_GET(rl, int64_t, nrow + 1, false);
    NL_GET(roff, int64_t, nrow + 1, false);
    k_row_count<<<nblk(nrow + 1), kNT>>>(nrow, ysf, ysn, lidx, leaves, t_nprt, rl);
    if ((st = scan(rl, roff, nrow + 1))) return st;
    int64_t nred_off = 0;
    if ((st = last(roff, nrow, nred_off))) return st;
    if (nred_off >= (int64_t(1) << 31)) return (err = "device near lists: too many scratch rows", -5);
    uint32_t *rk, *rk2;
    int64_t *rv, *red_off;
    int32_t* rc;
    NL_GET(rk, uint32_t, nred_off, false);
    NL_GET(rk2, uint32_t, nred_off, false);
    NL_GET(rv, int64_t, nred_off, false);
    NL_GET(red_off, int64_t, nred_off, true);
    NL_GET(rc, int32_t, nleaf + 1, false);
    NL_CK(cudaMemset(rc, 0, (size_t)(nleaf + 1) * 4));
    if (nrow) k_row_emit<<<nblk(nrow), kNT>>>(nrow, ysf, ysn, ysoff, lidx, leaves, t_nprt, roff, rk, rv, rc);
    NL_CK(cudaGetLastError());
    if (nred_off && (st = sort(rk, rk2, rv, red_off, nred_off, bits_for(nleaf)))) return st;
    int32_t *rf, *rfs, *red_first, *red_n;
    int64_t *rc64, *rcs, *red_ptr;
    NL_GET(rf, int32_t, nleaf + 1, false);
    NL_GET(rfs, int32_t, nleaf + 1, false);
    NL_GET(rc64, int64_t, nleaf + 1, false);
    NL_GET(rcs, int64_t, nleaf + 1, false);
    k_red_flags<<<nblk(nleaf + 1), kNT>>>(nleaf, rc, rf, rc64);
    if ((st = scan(rf, rfs, nleaf + 1)) || (st = scan(rc64, rcs, nleaf + 1))) return st;
    int32_t nred = 0;
    if ((st = last(rfs, nleaf, nred))) return st;
    NL_GET(red_first, int32_t, nred, true);
    NL_GET(red_n, int32_t, nred, true);
    NL_GET(red_ptr, int64_t, nred + 1, true);
    NL_CK(cudaMemset(red_ptr, 0, 8));
    if (nleaf) k_red_fill<<<nblk(nleaf), kNT>>>(nleaf, rc, rfs, rcs, leaves, t_first, t_nprt, red_first, red_n, red_ptr);
    NL_CK(cudaGetLastError());
    o.n_red = nred;
    o.red_first = red_first;
    o.red_n = red_n;
    o.red_ptr = red_ptr;
    o.red_off = red_off;

    // 6. symmetric blocks cut into work items (lanes per source by chunk)
    Items y;
    if ((st = split(sym_cptr, ysf, ysn, ysoff, tn, y))) return st;
    o.sym_items = y.n;
    o.sym_ptr = y.ptr;
    o.sym_sfirst = y.sf;
    o.sym_sn = y.sn;
    o.sym_soff = y.soff;
    o.sym_item_chunk = y.chunk;
    o.sym_chunk_items = y.chunk_items;
    o.sym_order = y.order;
  }

  // 7. every chunk's ranges cut into work items (the target-side near field)
  Items it;
  if ((st = split(rptr, rsf, rsn, nullptr, nullptr, it))) return st;
  o.p2p_items = it.n;
  o.p2p_ptr = it.ptr;
  o.p2p_sfirst = it.sf;
  o.p2p_sn = it.sn;
  o.p2p_item_chunk = it.chunk;
  o.p2p_chunk_items = it.chunk_items;
  o.p2p_order = it.order;
  NL_CK(cudaDeviceSynchronize());
  o.on = true;
  p.dev_near_allocs.insert(p.dev_near_allocs.end(), M.out.begin(), M.out.end());
  M.out.clear();
  return 0;
}

}  // namespace dfb
