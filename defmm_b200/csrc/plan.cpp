// Host-side plan builder: see plan.hpp.
//
// Construction is level-wise and multi-threaded.  Where the reference's result
// is discrete (cells, admissibility, cones, effective directions) the
// floating-point operations are the reference's, in the reference's order, so
// the outcome is bit-identical; this file is compiled with FMA contraction off.
#include "plan.hpp"
#include "fp64_math.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <tuple>

namespace dfb {

void dft_twiddles(int P, double* w) {
  for (int m = 0; m < P; m++) {
    const long double a = 2.0L * 3.14159265358979323846264338327950288L * m / P;
    w[2 * m] = (double)cosl(a);
    w[2 * m + 1] = -(double)sinl(a);
  }
}

double node_coord(int i, int L, double alpha) {  // thetis_polynomials.hpp:126
  return alpha * (-1. + 2. * ((double)i / (double)(L - 1)));
}

namespace {

unsigned hw_threads() {
  static unsigned n = std::max(1u, std::thread::hardware_concurrency());
  return n;
}

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Dynamic-chunk parallel loop over [0, n).
template <typename F>
void pfor(int64_t n, int64_t grain, F f) {
  if (n <= 0) return;
  unsigned nt = hw_threads();
  if (nt == 1 || n <= grain) {
    for (int64_t i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<int64_t> next(0);
  auto work = [&]() {
    for (;;) {
      int64_t b = next.fetch_add(grain);
      if (b >= n) return;
      int64_t e = std::min(n, b + grain);
      for (int64_t i = b; i < e; i++) f(i);
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; t++) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}

// Run f(k, begin, end) on K contiguous chunks of [0, n) in parallel.
template <typename F>
void pchunks(int64_t n, int K, F f) {
  std::vector<std::thread> th;
  for (int k = 0; k < K; k++) {
    int64_t b = n * k / K, e = n * (k + 1) / K;
    th.emplace_back([&f, k, b, e]() { f(k, b, e); });
  }
  for (auto& t : th) t.join();
}

// Stable counting sort of [0, n) by key(k) in [0, m): ptr gets the m + 1
// bucket offsets and put(pos, k) places every k, ties in index order.  K
// contiguous blocks count and place in parallel, so the result is the
// serial one.
template <typename Key, typename Put>
void bucket_sort(int64_t n, int64_t m, std::vector<int64_t>& ptr, Key key, Put put) {
  const int K = (int)std::max<int64_t>(1, std::min<int64_t>(std::min<unsigned>(hw_threads(), 32), n / 65536 + 1));
  std::vector<std::vector<int64_t>> kc(K, std::vector<int64_t>(m, 0));
  pchunks(n, K, [&](int k, int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) kc[k][key(i)]++;
  });
  ptr.assign(m + 1, 0);
  for (int64_t c = 0; c < m; c++) {
    int64_t t = ptr[c];
    for (int k = 0; k < K; k++) {
      const int64_t v = kc[k][c];
      kc[k][c] = t;
      t += v;
    }
    ptr[c + 1] = t;
  }
  pchunks(n, K, [&](int k, int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) put(kc[k][key(i)]++, i);
  });
}

inline double norm3(const double* v) {
  double t = 0.;
  for (int i = 0; i < 3; i++) t += v[i] * v[i];
  return std::sqrt(t);
}

// --------------------------------------------------------------- octrees --
struct Node {
  int64_t first, n;
  double ctr[3], rad;
  int32_t idx[3], lvl;
  int64_t parent;
  int64_t child0 = 0;
  int nchild = 0;
  int64_t size = 1;   // subtree cell count
  int64_t dfs = 0;    // depth-first index
};

// Level-wise build of the reference's octree (sort.hpp:98-228): a cell splits
// into the non-empty octants of bit code sum_k (x_k > c_k) << k unless it is
// a leaf (fewer than ncrit particles, sort.hpp:49, or lvl >= lvmax with
// lvmax >= 0, sort.hpp:51); child centres c + (r/2)(2 b_k - 1); particles are
// split stably, so a leaf keeps the input order of its particles.
int build_tree(Tree& t, const double* pts, int64_t n, const double* bctr,
               double brad, int ncrit, int lvmax, std::string& err, TreeSorter* sorter) {
  std::vector<int32_t> order(sorter ? 0 : n);
  for (int64_t i = 0; i < (int64_t)order.size(); i++) order[i] = (int32_t)i;
  std::vector<int32_t> tmp(sorter ? 0 : n);
  if (sorter) {
    const int st = sorter->begin(pts, n, err);
    if (st) return st;
  }
  std::vector<Node> nodes(1);
  Node& r = nodes[0];
  r.first = 0;
  r.n = n;
  for (int k = 0; k < 3; k++) {
    r.ctr[k] = bctr[k];
    r.idx[k] = 0;
  }
  r.rad = brad;
  r.lvl = 0;
  r.parent = -1;
  int64_t lb = 0, le = 1;
  int lvl = 0;
  while (lb < le) {
    const int64_t cnt = le - lb;
    std::vector<std::array<int64_t, 8>> hist(cnt);
    std::atomic<int> bad(0);
    if (sorter) {  // octant counts on the sorter's side
      std::vector<int64_t> first(cnt);
      std::vector<double> ctr(3 * cnt);
      std::vector<uint8_t> split(cnt);
      for (int64_t ii = 0; ii < cnt; ii++) {
        const Node& c = nodes[lb + ii];
        first[ii] = c.first;
        for (int k = 0; k < 3; k++) ctr[3 * ii + k] = c.ctr[k];
        const bool stop = lvmax >= 0 ? c.lvl >= lvmax : c.n < ncrit;
        split[ii] = stop ? 0 : 1;
        if (!stop && c.lvl >= 60) bad = 1;
      }
      if (bad) {
        err = "coincident points keep a cell at or above the leaf size beyond level 60";
        return -2;
      }
      std::vector<int64_t> hflat(8 * cnt, 0);
      const int st = sorter->histogram(cnt, first.data(), ctr.data(), split.data(), hflat.data(), err);
      if (st) return st;
      for (int64_t ii = 0; ii < cnt; ii++)
        for (int b = 0; b < 8; b++) hist[ii][b] = hflat[8 * ii + b];
    } else
    pfor(cnt, 1, [&](int64_t ii) {
      Node& c = nodes[lb + ii];
      auto& h = hist[ii];
      h.fill(0);
      const bool stop = lvmax >= 0 ? c.lvl >= lvmax : c.n < ncrit;
      if (stop) return;
      if (c.lvl >= 60) {
        bad = 1;
        return;
      }
      std::vector<uint8_t> code(c.n);
      for (int64_t i = 0; i < c.n; i++) {
        const double* p = pts + 3 * (int64_t)order[c.first + i];
        int b = 0;
        for (int k = 0; k < 3; k++) b += ((p[k] > c.ctr[k]) ? 1 : 0) << k;
        code[i] = (uint8_t)b;
        h[b]++;
      }
      int64_t off[8], add[8] = {0};
      off[0] = 0;
      for (int b = 1; b < 8; b++) off[b] = off[b - 1] + h[b - 1];
      for (int64_t i = 0; i < c.n; i++) {
        int b = code[i];
        tmp[c.first + off[b] + add[b]++] = order[c.first + i];
      }
      std::memcpy(&order[c.first], &tmp[c.first], sizeof(int32_t) * c.n);
    });
    if (bad) {
      err = "coincident points keep a cell at or above the leaf size beyond level 60";
      return -2;
    }
    // create the children of this level, in octant order per parent
    int64_t total = 0;
    for (int64_t ii = 0; ii < cnt; ii++) {
      Node& c = nodes[lb + ii];
      c.child0 = le + total;
      int k = 0;
      for (int b = 0; b < 8; b++) k += hist[ii][b] ? 1 : 0;
      c.nchild = k;
      total += k;
    }
    nodes.resize(le + total);
    pfor(cnt, 64, [&](int64_t ii) {
      Node& c = nodes[lb + ii];
      if (!c.nchild) return;
      const double nrad = c.rad / 2.;
      int64_t off = 0, ch = c.child0;
      for (int b = 0; b < 8; b++) {
        int64_t h = hist[ii][b];
        if (!h) continue;
        Node& s = nodes[ch++];
        s.first = c.first + off;
        s.n = h;
        for (int k = 0; k < 3; k++) {
          s.ctr[k] = c.ctr[k] + nrad * (double)(((b >> k) & 1) * 2 - 1);
          s.idx[k] = 2 * c.idx[k] + ((b >> k) & 1);
        }
        s.rad = nrad;
        s.lvl = c.lvl + 1;
        s.parent = lb + ii;
        off += h;
      }
    });
    if (sorter && total) {  // children's ranges: the sorter moves the particles
      std::vector<int64_t> cf(8 * cnt, -1);
      for (int64_t ii = 0; ii < cnt; ii++) {
        const Node& c = nodes[lb + ii];
        int64_t ch = c.child0;
        for (int b = 0; b < 8; b++)
          if (hist[ii][b]) cf[8 * ii + b] = nodes[ch++].first;
      }
      const int st = sorter->reorder(cf.data(), err);
      if (st) return st;
    }
    lb = le;
    le = le + total;
    lvl++;
  }
  if (sorter) {
    order.resize(n);
    const int st = sorter->finish(order.data(), err);
    if (st) return st;
  }
  const int64_t nc = (int64_t)nodes.size();
  // subtree sizes bottom-up (children always follow their parent in BFS order)
  for (int64_t i = nc - 1; i > 0; i--) nodes[nodes[i].parent].size += nodes[i].size;
  // depth-first pre-order numbering, children in octant order
  nodes[0].dfs = 0;
  for (int64_t i = 0; i < nc; i++) {
    int64_t d = nodes[i].dfs + 1;
    for (int j = 0; j < nodes[i].nchild; j++) {
      Node& s = nodes[nodes[i].child0 + j];
      s.dfs = d;
      d += s.size;
    }
  }
  t.ncell = nc;
  t.idx.resize(3 * nc);
  t.lvl.resize(nc);
  t.nprt.resize(nc);
  t.first.resize(nc);
  t.parent.resize(nc);
  t.nson.resize(nc);
  t.sub_end.resize(nc);
  t.ctr.resize(3 * nc);
  t.rad.resize(nc);
  int maxl = 0;
  for (int64_t i = 0; i < nc; i++) {
    const Node& c = nodes[i];
    int64_t d = c.dfs;
    for (int k = 0; k < 3; k++) {
      t.idx[3 * d + k] = c.idx[k];
      t.ctr[3 * d + k] = c.ctr[k];
    }
    t.lvl[d] = c.lvl;
    t.nprt[d] = (int32_t)c.n;
    t.first[d] = (int32_t)c.first;
    t.parent[d] = c.parent < 0 ? -1 : (int32_t)nodes[c.parent].dfs;
    t.nson[d] = c.nchild;
    t.sub_end[d] = (int32_t)(d + c.size);
    t.rad[d] = c.rad;
    maxl = std::max(maxl, c.lvl);
  }
  t.son_ptr.assign(nc + 1, 0);
  for (int64_t d = 0; d < nc; d++) t.son_ptr[d + 1] = t.son_ptr[d] + t.nson[d];
  t.sons.resize(t.son_ptr[nc]);
  for (int64_t i = 0; i < nc; i++) {
    const Node& c = nodes[i];
    for (int j = 0; j < c.nchild; j++)
      t.sons[t.son_ptr[c.dfs] + j] = (int32_t)nodes[c.child0 + j].dfs;
  }
  t.nlvl = maxl + 1;
  t.lvl_cells.assign(t.nlvl, 0);
  for (int64_t d = 0; d < nc; d++) t.lvl_cells[t.lvl[d]]++;
  t.perm = order;
  t.pos.resize(3 * n);
  for (int64_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) t.pos[3 * i + k] = pts[3 * (int64_t)order[i] + k];
  return 0;
}

// ----------------------------------------------------- frequency regime --
// frequency.hpp:44-184: cpt halvings until kappa*diam <= 1 (eta = 1); levels
// l <= cpt are HF with direction stage cpt - l and 6*4^stage directions;
// M2L and the up/down operators run from the first level s >= 2 at which
// kappa*2R/4^s <= 1.
int init_levels(Plan& p, std::string& err) {
  Levels& v = p.lv;
  v.nlvl = std::max(p.S.nlvl, p.T.nlvl);
  double diam = 2. * p.box_rad;
  int cpt = 0;
  if (diam * p.kappa > 1.) {
    while (diam * p.kappa > 1.) {
      diam /= 2.;
      cpt++;
    }
  }
  v.cpt = cpt;
  v.noHF = !(cpt > 1);
  v.isHF.assign(v.nlvl, 0);
  v.HFStage.assign(v.nlvl, 0);
  for (int l = std::min(cpt, v.nlvl - 1); l >= 0; l--) {
    v.isHF[l] = cpt - l + 1;
    v.HFStage[l] = cpt - l;
  }
  v.nDir.assign(v.nlvl, 1);
  for (int l = 1; l < v.nlvl; l++)
    if (v.isHF[l]) v.nDir[l] = 6 << (2 * v.HFStage[l]);
  int ms = 0;
  const double bd = 2. * p.box_rad;
  while (1. < p.kappa * bd / (double)(1 << ms) / (double)(1 << ms)) {
    ms++;
    if (ms >= v.nlvl) {
      err = "tree too shallow: no level admits precomputed far-field interactions";
      return -3;
    }
  }
  v.max_stage = std::max(ms, 2);
  v.prec.assign(v.nlvl, 0);
  for (int l = v.max_stage; l < v.nlvl; l++) v.prec[l] = 1;
  v.nCellMax.assign(v.nlvl, -1);
  for (int l = 0; l < v.nlvl; l++) {
    if (!v.prec[l]) continue;
    v.nCellMax[l] = v.isHF[l] ? (1 << l) : (v.isHF[l - 1] ? 8 : 4);
  }
  return 0;
}

// ------------------------------------------------------------ directions --
// newdirections.hpp:76-171.  Stage e holds 6 blocks of 4^e directions: the
// +x face refined from stage e-1 (its block 0) by offsets (0, +-r, +-r),
// r = 2^-(e+1), then normalised; block 1 its mirror image x -> -x; blocks
// 2-3 and 4-5 the cyclic rotations d_k <- src_{(k+1)%3} and d_k <-
// src_{(k+2)%3} of blocks 0-1.  Stage 0 is +x,-x,+y,-y,+z,-z.
void init_directions(Plan& p) {
  const int ns = p.lv.cpt;
  p.dirs.assign(ns, {});
  if (!ns) return;
  for (int e = 0; e < ns; e++) p.dirs[e].assign(3 * ((size_t)6 << (2 * e)), 0.);
  for (int k = 0; k < 3; k++) {
    p.dirs[0][3 * (2 * k) + k] = 1.;
    p.dirs[0][3 * (2 * k + 1) + k] = -1.;
  }
  int64_t face = 1;  // 4^(e-1) directions on the +x face of stage e-1
  for (int e = 1; e < ns; e++) {
    const double r = 1. / (double)(1 << (e + 1));
    for (int64_t i = 0; i < face; i++)
      for (int q = 0; q < 4; q++) {
        const double off[3] = {0., (q & 1) ? -1. : 1., (q & 2) ? -1. : 1.};
        double d[3];
        for (int k = 0; k < 3; k++) d[k] = p.dirs[e - 1][3 * i + k] + off[k] * r;
        const double nr = norm3(d);
        for (int k = 0; k < 3; k++) p.dirs[e][3 * (4 * i + q) + k] = d[k] / nr;
      }
    face *= 4;
    const int64_t fs = face;  // 4^e
    for (int64_t j = 0; j < fs; j++) {
      for (int k = 0; k < 3; k++) p.dirs[e][3 * (fs + j) + k] = p.dirs[e][3 * j + k];
      p.dirs[e][3 * (fs + j)] *= -1.;
    }
    for (int rot = 1; rot < 3; rot++)
      for (int64_t j = 0; j < 2 * fs; j++)
        for (int k = 0; k < 3; k++)
          p.dirs[e][3 * (rot * 2 * fs + j) + k] = p.dirs[e][3 * j + (k + rot) % 3];
  }
}

// newdirections.hpp:175-185: the direction nearest to u, lowest index on ties
int nearest_direction(const std::vector<double>& tab, const double* u) {
  double best = 1.e30;
  int ind = -1;
  const int n = (int)(tab.size() / 3);
  for (int i = 0; i < n; i++) {
    const double df[3] = {tab[3 * i] - u[0], tab[3 * i + 1] - u[1], tab[3 * i + 2] - u[2]};
    const double d = norm3(df);
    if (best > d) {
      best = d;
      ind = i;
    }
  }
  return ind;
}

// ---------------------------------------------- polynomials and symmetries --
inline void unflatten(int i, int n, int* I) {
  I[2] = i % n;
  I[1] = (i / n) % n;
  I[0] = i / (n * n);
}
inline double node1d(int i, int L, double alpha) {  // thetis_polynomials.hpp:126
  return alpha * (-1. + 2. * ((double)i / (double)(L - 1)));
}
// equispaced Lagrange basis function i of order P on [-alpha, alpha]
// (thetis_polynomials.hpp:81-94)
double lagrange(int i, double x, int P, double alpha) {
  double res = 1., nx = x / alpha;
  const double pi = -1. + 2. * ((double)i / (double)(P - 1));
  for (int j = 0; j < P; j++) {
    if (j == i) continue;
    const double pj = -1. + 2. * ((double)j / (double)(P - 1));
    res *= (nx - pj) / (pi - pj);
  }
  return res;
}

// hypercube symmetry of a translation (hypercube.hpp:109-136,
// permutations.hpp:88-120, :209-232): axis order code, sign code, and the
// fundamental index (|iZ| permuted into non-increasing order)
const int kAxisOrder[8][3] = {{0, 1, 2}, {1, 0, 2}, {0, 1, 2}, {1, 2, 0},
                              {0, 2, 1}, {0, 1, 2}, {2, 0, 1}, {2, 1, 0}};
inline void symmetry(const int* iZ, int* nI, int& hsh) {
  const int a0 = std::abs(iZ[0]), a1 = std::abs(iZ[1]), a2 = std::abs(iZ[2]);
  const int h1 = (a0 < a1 ? 1 : 0) | (a0 < a2 ? 2 : 0) | (a1 < a2 ? 4 : 0);
  const int h0 = (iZ[0] < 0 ? 1 : 0) | (iZ[1] < 0 ? 2 : 0) | (iZ[2] < 0 ? 4 : 0);
  for (int k = 0; k < 3; k++) nI[k] = std::abs(iZ[kAxisOrder[h1][k]]);
  hsh = h0 + (h1 << 3);
}

void init_small_tables(Plan& p) {
  const int L = p.L, P = p.P;
  // circulant.hpp:47-93
  p.itilda.resize(p.LL);
  for (int i = 0; i < p.LL; i++) {
    int I[3];
    unflatten(i, L, I);
    p.itilda[i] = (I[0] * P + I[1]) * P + I[2];
  }
  p.tabZ.resize(3 * p.PP);
  for (int i = 0; i < p.PP; i++) {
    int E[3];
    unflatten(i, P, E);
    for (int k = 0; k < 3; k++) {
      const int e = E[k] < L ? E[k] : -(2 * L - 1 - E[k]);
      p.tabZ[3 * i + k] = node1d(e > -1 ? e : 0, L, 1.) - node1d(e > -1 ? 0 : -e, L, 1.);
    }
  }
  // permutations.hpp:128-150: spectrum index map of each of the 64 codes
  p.perm.resize(64 * (size_t)p.PP);
  for (int h0 = 0; h0 < 8; h0++)
    for (int h1 = 0; h1 < 8; h1++) {
      const int h = h0 + (h1 << 3);
      for (int i = 0; i < p.PP; i++) {
        int tp[3], tm[3];
        unflatten(i, P, tp);
        for (int k = 0; k < 3; k++) {
          const int ax = kAxisOrder[h1][k];
          tm[k] = tp[ax];
          if ((h0 & (1 << ax)) && tm[k]) tm[k] = P - tm[k];
        }
        p.perm[(size_t)h * p.PP + i] = (uint16_t)((tm[0] * P + tm[1]) * P + tm[2]);
      }
    }
  // interpolation.hpp:184-242: parent basis k at child node p, child on the
  // negative (0) or positive (1) side
  for (int sg = 0; sg < 2; sg++) {
    p.m2m[sg].assign(L * L, 0.);
    p.l2l[sg].assign(L * L, 0.);
    for (int q = 0; q < L; q++)
      for (int k = 0; k < L; k++) {
        const double v = lagrange(k, node1d(q, L, 1.) + (sg ? 1. : -1.), L, 2.);
        p.m2m[sg][k + q * L] = v;
        p.l2l[sg][q + k * L] = v;
      }
  }
}

// planewave.hpp:44-69: sig = exp(-i kappa d.x) on the grid of radius R/2^(l+1)
// and its square (the grid of radius R/2^l)
// values = false: the sizes only (the device fills the values)
void init_signatures(Plan& p, bool values) {
  const Levels& v = p.lv;
  p.sig.assign(std::max(1, v.cpt + 1), {});
  p.sig2.assign(std::max(1, v.cpt + 1), {});
  for (int l = 2; l < v.nlvl; l++) {
    if (!(v.prec[l] && v.isHF[l])) continue;
    const int h = v.HFStage[l];
    const double locrad = p.box_rad / (double)(1 << l);
    const int nd = v.nDir[l];
    auto& s1 = p.sig[h];
    auto& s2 = p.sig2[h];
    s1.resize((size_t)nd * p.LL);
    s2.resize((size_t)nd * p.LL);
    if (!values) continue;
    pfor(nd, 16, [&](int64_t d) {
      const double* dv = &p.dirs[h][3 * d];
      for (int k = 0; k < p.LL; k++) {
        int I[3];
        unflatten(k, p.L, I);
        double dp = 0.;
        for (int a = 0; a < 3; a++) dp += dv[a] * node1d(I[a], p.L, .5 * locrad);
        const double ang = p.kappa * dp;
        double sn, cs;
        sincos_fp64(ang, sn, cs);
        const cplx s(cs, -sn);
        s1[d * p.LL + k] = s;
        s2[d * p.LL + k] = s * s;
      }
    });
  }
}

// Unnormalised forward 3-D DFT of size P (row-major), FP64, by definition.
void dft3(cplx* x, int P) {
  std::vector<cplx> w(P), line(P), res(P);
  std::vector<double> wt(2 * P);
  dft_twiddles(P, wt.data());
  for (int m = 0; m < P; m++) w[m] = cplx(wt[2 * m], wt[2 * m + 1]);
  int inner = 1;
  for (int d = 2; d >= 0; d--) {
    const int outer = P * P / inner;
    for (int o = 0; o < outer; o++)
      for (int i = 0; i < inner; i++) {
        cplx* b = x + (int64_t)o * P * inner + i;
        for (int j = 0; j < P; j++) line[j] = b[j * inner];
        for (int k = 0; k < P; k++) {
          cplx acc = 0.;
          for (int j = 0, m = 0; j < P; j++, m = (m + k) % P) acc += line[j] * w[m];
          res[k] = acc;
        }
        for (int k = 0; k < P; k++) b[k * inner] = res[k];
      }
    inner *= P;
  }
}

// circulant.hpp:133-144: spectrum of the kernel sampled on the circulant grid
// of the translation v = 2 nI r
void transfer_spectrum(const Plan& p, double rad, const int* nI, cplx* out) {
  double v[3];
  for (int k = 0; k < 3; k++) v[k] = 2. * (double)nI[k] * rad;
  for (int i = 0; i < p.PP; i++) {
    double z[3];
    for (int k = 0; k < 3; k++) z[k] = v[k] + p.tabZ[3 * i + k] * rad;
    const double R = norm3(z);
    const double a = R * p.kappa;
    double sn, cs;
    sincos_fp64(a, sn, cs);
    out[i] = cplx(cs, sn) / (4. * M_PI * R);
  }
  dft3(out, p.P);
}

// admissibility: hrzpass.hpp:40-49 (MAClist), :52-56 (MACgeomhf)
inline bool adm_lf(const Tree& T, int64_t t, const Tree& S, int64_t s) {
  int test = 0, ncmp = 3;
  for (int k = 0; k < 3; k++) {
    const int d = T.idx[3 * t + k] - S.idx[3 * s + k];
    ncmp -= d ? 0 : 1;
    test += std::abs(d);
  }
  return test > ncmp;
}
inline bool adm_hf(const Tree& T, int64_t t, const Tree& S, int64_t s, double kappa) {
  const double d[3] = {T.ctr[3 * t] - S.ctr[3 * s], T.ctr[3 * t + 1] - S.ctr[3 * s + 1],
                       T.ctr[3 * t + 2] - S.ctr[3 * s + 2]};
  const double tmp = (1. - 1.e-8) * (norm3(d) - 2. * S.rad[s]);
  const double tt = 2. * S.rad[s];
  return tmp >= std::max(tt * tt * kappa, tt);
}

}  // namespace

int64_t Slots::slot_of(int64_t c, int d) const {
  const int64_t b = cell_ptr[c], e = cell_ptr[c + 1];
  if (b == e) return -1;
  if (d < 0) return cell_dirs[b] < 0 ? cell_slots[b] : -1;
  auto it = std::lower_bound(cell_dirs.begin() + b, cell_dirs.begin() + e, d);
  if (it == cell_dirs.begin() + e || *it != d) return -1;
  return cell_slots[it - cell_dirs.begin()];
}

namespace {

// Per-level state while walking the dual tree top-down.
struct LevelFlags {
  std::vector<int64_t> cells;        // cells of the level, DFS order
  std::vector<uint8_t> eff;          // cells.size() x nDir
};

// Assign slots for one tree at one level, cone-major (see Slots).
void level_slots(const Plan& p, int l, const LevelFlags& F, Slots& s,
                 std::vector<int32_t>& dense) {
  const Levels& v = p.lv;
  const int64_t nc = (int64_t)F.cells.size();
  if (!v.prec[l]) {
    s.cone_begin[l].assign(2, s.n);
    return;
  }
  if (!v.isHF[l]) {  // one LF expansion per cell
    s.cone_begin[l] = {s.n, s.n + nc};
    for (int64_t i = 0; i < nc; i++) {
      s.cell.push_back((int32_t)F.cells[i]);
      s.dir.push_back(-1);
    }
    dense.assign(nc, 0);
    for (int64_t i = 0; i < nc; i++) dense[i] = (int32_t)(s.n + i);
    s.n += nc;
    return;
  }
  const int nd = v.nDir[l];
  std::vector<int64_t> cnt(nd, 0);
  pfor(nd, 4, [&](int64_t d) {
    int64_t c = 0;
    for (int64_t i = 0; i < nc; i++) c += F.eff[i * nd + d];
    cnt[d] = c;
  });
  s.cone_begin[l].assign(nd + 1, 0);
  s.cone_begin[l][0] = s.n;
  for (int d = 0; d < nd; d++) s.cone_begin[l][d + 1] = s.cone_begin[l][d] + cnt[d];
  const int64_t tot = s.cone_begin[l][nd] - s.n;
  const int64_t base = s.n;
  s.cell.resize(base + tot);
  s.dir.resize(base + tot);
  dense.assign(nc * nd, -1);
  pfor(nd, 4, [&](int64_t d) {
    int64_t k = s.cone_begin[l][d];
    for (int64_t i = 0; i < nc; i++)
      if (F.eff[i * nd + d]) {
        s.cell[k] = (int32_t)F.cells[i];
        s.dir[k] = (int32_t)d;
        dense[i * nd + d] = (int32_t)k;
        k++;
      }
  });
  s.n += tot;
}

// Symmetric decomposition of the near field (Plan::self_*, sym_*, red_*),
// for one tree holding both sources and targets.  Source ranges are unions
// of whole leaves, and a leaf's own range is always present (its self pair).
// Scratch is chunk-major: a chunk's symmetric ranges take consecutive slots.
// Indices 0..n-1 ordered by decreasing key, ties in index order (the order
// of a stable sort by key > key): a counting sort when the keys are small,
// else a stable sort.
std::vector<int32_t> order_by_decreasing(const std::vector<int64_t>& key) {
  const int64_t n = (int64_t)key.size();
  std::vector<int32_t> order(n);
  int64_t kmax = 0;
  for (int64_t k : key) kmax = std::max(kmax, k);
  if (kmax >= 0 && kmax <= std::max<int64_t>(1 << 20, 4 * n)) {
    std::vector<int64_t> start(kmax + 2, 0);
    for (int64_t k : key) start[kmax - std::max<int64_t>(k, 0) + 1]++;  // bucket of key k: kmax - k
    for (int64_t b = 0; b <= kmax; b++) start[b + 1] += start[b];
    for (int64_t i = 0; i < n; i++) order[start[kmax - std::max<int64_t>(key[i], 0)]++] = (int32_t)i;
    return order;
  }
  for (int64_t i = 0; i < n; i++) order[i] = (int32_t)i;
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return key[a] > key[b]; });
  return order;
}

void build_symmetric_near(Plan& p) {
  const Tree& T = p.T;
  const int64_t nch = (int64_t)p.p2p_tfirst.size();
  std::vector<int32_t> leaf_at(T.pos.size() / 3, -1);  // particle -> leaf
  pfor(T.ncell, 1024, [&](int64_t c) {
    if (T.leaf(c))
      for (int32_t k = 0; k < T.nprt[c]; k++) leaf_at[T.first[c] + k] = (int32_t)c;
  });
  // per chunk: own-leaf blocks, blocks of the source leaves after the own
  // leaf and their sources; then prefix sums and a parallel fill, in chunk
  // order (the serial order of the lists)
  std::vector<int64_t> nself(nch + 1, 0), nsym(nch + 1, 0), nsrc(nch + 1, 0);
  pfor(nch, 256, [&](int64_t ch) {
    const int32_t lf = leaf_at[p.p2p_tfirst[ch]];
    const int32_t a0 = T.first[lf], a1 = a0 + T.nprt[lf];
    for (int64_t r = p.p2p_ptr[ch]; r < p.p2p_ptr[ch + 1]; r++) {
      const int32_t s0 = p.p2p_sfirst[r], s1 = s0 + p.p2p_sn[r];
      if (s0 < a1 && s1 > a0) nself[ch + 1]++;
      const int32_t b0 = std::max(s0, a1);
      if (b0 < s1) {
        nsym[ch + 1]++;
        nsrc[ch + 1] += s1 - b0;
      }
    }
  });
  for (int64_t ch = 0; ch < nch; ch++) {
    nself[ch + 1] += nself[ch];
    nsym[ch + 1] += nsym[ch];
    nsrc[ch + 1] += nsrc[ch];
  }
  p.self_ptr.assign(nself.begin(), nself.end());
  p.sym_ptr.assign(nsym.begin(), nsym.end());
  p.self_sfirst.assign(nself[nch], 0);
  p.self_sn.assign(nself[nch], 0);
  p.sym_sfirst.assign(nsym[nch], 0);
  p.sym_sn.assign(nsym[nch], 0);
  p.sym_soff.assign(nsym[nch], 0);
  pfor(nch, 256, [&](int64_t ch) {
    const int32_t lf = leaf_at[p.p2p_tfirst[ch]];
    const int32_t a0 = T.first[lf], a1 = a0 + T.nprt[lf];
    int64_t ks = nself[ch], ky = nsym[ch], tot = nsrc[ch];
    for (int64_t r = p.p2p_ptr[ch]; r < p.p2p_ptr[ch + 1]; r++) {
      const int32_t s0 = p.p2p_sfirst[r], s1 = s0 + p.p2p_sn[r];
      if (s0 < a1 && s1 > a0) {  // the own leaf
        p.self_sfirst[ks] = a0;
        p.self_sn[ks++] = a1 - a0;
      }
      const int32_t b0 = std::max(s0, a1);
      if (b0 < s1) {  // source leaves after the own leaf
        p.sym_sfirst[ky] = b0;
        p.sym_sn[ky] = s1 - b0;
        p.sym_soff[ky++] = tot;
        tot += s1 - b0;
      }
    }
  });
  p.sym_scratch = nsrc[nch];
  // rows per source leaf, in row order: each of K contiguous blocks of rows
  // counts its rows per leaf, so that its rows land after those of the
  // blocks before it
  const int64_t nrow = (int64_t)p.sym_sfirst.size();
  const int K = (int)std::max<int64_t>(1, std::min<int64_t>(std::min<unsigned>(hw_threads(), 32), nrow / 4096 + 1));
  std::vector<std::vector<int64_t>> kc(K, std::vector<int64_t>(T.ncell, 0));
  auto each_leaf = [&](int64_t r, auto f) {
    for (int32_t j = p.sym_sfirst[r]; j < p.sym_sfirst[r] + p.sym_sn[r]; j += T.nprt[leaf_at[j]]) f(leaf_at[j], j);
  };
  pchunks(nrow, K, [&](int k, int64_t b, int64_t e) {
    for (int64_t r = b; r < e; r++) each_leaf(r, [&](int32_t c, int32_t) { kc[k][c]++; });
  });
  p.red_first.clear();
  p.red_n.clear();
  p.red_ptr.assign(1, 0);
  for (int64_t c = 0; c < T.ncell; c++) {
    int64_t n = 0;
    for (int k = 0; k < K; k++) {
      const int64_t v = kc[k][c];
      kc[k][c] = n;  // rows of the blocks before k
      n += v;
    }
    if (n) {
      for (int k = 0; k < K; k++) kc[k][c] += p.red_ptr.back();
      p.red_first.push_back(T.first[c]);
      p.red_n.push_back(T.nprt[c]);
      p.red_ptr.push_back(p.red_ptr.back() + n);
    }
  }
  p.red_off.assign(p.red_ptr.back(), 0);
  pchunks(nrow, K, [&](int k, int64_t b, int64_t e) {
    for (int64_t r = b; r < e; r++)
      each_leaf(r, [&](int32_t c, int32_t j) { p.red_off[kc[k][c]++] = p.sym_soff[r] + (j - p.sym_sfirst[r]); });
  });
  // self blocks by decreasing work
  std::vector<int64_t> ws(nch, 0);
  pfor(nch, 1024, [&](int64_t ch) {
    for (int64_t r = p.self_ptr[ch]; r < p.self_ptr[ch + 1]; r++) ws[ch] += p.self_sn[r];
  });
  p.self_order.clear();
  for (int32_t ch : order_by_decreasing(ws))
    if (ws[ch]) p.self_order.push_back(ch);
}

// Cut every chunk's source ranges (CSR `ptr` over chunks) into items of at
// most kItemSources sources, in place: ptr becomes a CSR over items, ranges
// are split at item boundaries (with their scratch slots, if any); `chunk`
// maps items to chunks, `items` chunks to their consecutive items, and
// `order` lists items by decreasing work (sources x lanes per source).
void split_items(const Plan& p, std::vector<int64_t>& ptr, std::vector<int32_t>& sf, std::vector<int32_t>& sn,
                 std::vector<int64_t>* soff, std::vector<int32_t>& chunk, std::vector<int64_t>& items,
                 std::vector<int32_t>& order, bool lanes_by_chunk) {
  constexpr int64_t SP = Plan::kItemSources;
  const int64_t nch = (int64_t)ptr.size() - 1;
  // per chunk: items (ceil(sources / SP)) and range pieces (a range is cut
  // where an item ends); then prefix sums and a parallel fill in chunk order
  std::vector<int64_t> nit(nch + 1, 0), npc(nch + 1, 0);
  pfor(nch, 256, [&](int64_t ch) {
    int64_t fill = 0, pieces = 0, its = 0;
    for (int64_t r = ptr[ch]; r < ptr[ch + 1]; r++)
      for (int32_t o = 0; o < sn[r];) {
        const int32_t take = (int32_t)std::min<int64_t>(sn[r] - o, SP - fill);
        pieces++;
        fill += take;
        o += take;
        if (fill == SP) {
          its++;
          fill = 0;
        }
      }
    if (fill) its++;
    nit[ch + 1] = its;
    npc[ch + 1] = pieces;
  });
  for (int64_t ch = 0; ch < nch; ch++) {
    nit[ch + 1] += nit[ch];
    npc[ch + 1] += npc[ch];
  }
  const int64_t nitem = nit[nch], npiece = npc[nch];
  std::vector<int64_t> nptr(nitem + 1, 0);
  std::vector<int32_t> nsf(npiece), nsn(npiece);
  std::vector<int64_t> nso(soff ? npiece : 0);
  std::vector<int64_t> work(nitem);
  chunk.assign(nitem, 0);
  pfor(nch, 256, [&](int64_t ch) {
    int tp = 32;
    if (lanes_by_chunk) {
      tp = 4;
      while (tp < p.p2p_tn[ch]) tp <<= 1;
    }
    int64_t fill = 0, q = npc[ch], it = nit[ch];
    for (int64_t r = ptr[ch]; r < ptr[ch + 1]; r++)
      for (int32_t o = 0; o < sn[r];) {
        const int32_t take = (int32_t)std::min<int64_t>(sn[r] - o, SP - fill);
        nsf[q] = sf[r] + o;
        nsn[q] = take;
        if (soff) nso[q] = (*soff)[r] + o;
        q++;
        fill += take;
        o += take;
        if (fill == SP) {
          nptr[it + 1] = q;
          chunk[it] = (int32_t)ch;
          work[it++] = fill * tp;
          fill = 0;
        }
      }
    if (fill) {
      nptr[it + 1] = q;
      chunk[it] = (int32_t)ch;
      work[it++] = fill * tp;
    }
  });
  items.assign(nit.begin(), nit.end());
  ptr.swap(nptr);
  sf.swap(nsf);
  sn.swap(nsn);
  if (soff) soff->swap(nso);
  order = order_by_decreasing(work);
}

}  // namespace

// The level walk on the host (see LevelWalk): frontier pairs level by level
// in depth-first order, multi-threaded per level.
int walk_levels_host(Plan& p, LevelWalk& walk) {
  const Levels& v = p.lv;
  const int nlvl = v.nlvl;
  const double kappa = p.kappa;
  // per-level cell lists (DFS order) and level-local indices
  auto level_lists = [&](const Tree& tr, std::vector<std::vector<int64_t>>& lists,
                         std::vector<int32_t>& loc) {
    lists.assign(nlvl, {});
    loc.assign(tr.ncell, -1);
    for (int64_t c = 0; c < tr.ncell; c++) {
      loc[c] = (int32_t)lists[tr.lvl[c]].size();
      lists[tr.lvl[c]].push_back(c);
    }
  };
  std::vector<std::vector<int64_t>> lcT, lcS;
  std::vector<int32_t> locT, locS;
  level_lists(p.T, lcT, locT);
  level_lists(p.S, lcS, locS);

  p.sT = Slots();
  p.sS = Slots();
  p.sT.lvl_begin.assign(nlvl + 1, 0);
  p.sS.lvl_begin.assign(nlvl + 1, 0);
  p.sT.cone_begin.assign(nlvl, {});
  p.sS.cone_begin.assign(nlvl, {});

  // M2L entries per level before grouping by target slot
  walk.far_ts.assign(nlvl, {});
  walk.far_ss.assign(nlvl, {});
  walk.far_tab.assign(nlvl, {});
  auto& near_pairs = walk.near_pairs;
  auto& tab_nI = walk.tab_nI;
  near_pairs.clear();
  tab_nI.clear();
  std::vector<int32_t> denseT, denseS, denseT_prev, denseS_prev;
  LevelFlags fT_prev, fS_prev;
  int64_t table_count = 0;

  // frontier of the dual traversal (hrzpass.hpp:62-91), kept in the
  // reference's depth-first order
  std::vector<std::pair<int32_t, int32_t>> frontier{{0, 0}};
  const int K = (int)hw_threads();
  for (int l = 0; l < nlvl; l++) {
    // 1. classify this level's pairs: far (M2L), near (P2P) or split
    std::vector<std::vector<std::pair<int32_t, int32_t>>> c_far(K), c_near(K), c_next(K);
    const bool prec = v.prec[l], hf = l > 0 && v.isHF[l];
    pchunks((int64_t)frontier.size(), K, [&](int k, int64_t b, int64_t e) {
      for (int64_t i = b; i < e; i++) {
        const int32_t t = frontier[i].first, s = frontier[i].second;
        if (prec) {
          const bool adm = hf ? adm_hf(p.T, t, p.S, s, kappa) : adm_lf(p.T, t, p.S, s);
          if (adm) {
            c_far[k].push_back({t, s});
            continue;
          }
        }
        if (p.T.leaf(t) || p.S.leaf(s)) {
          c_near[k].push_back({t, s});
          continue;
        }
        for (int64_t a = p.T.son_ptr[t]; a < p.T.son_ptr[t + 1]; a++)
          for (int64_t bb = p.S.son_ptr[s]; bb < p.S.son_ptr[s + 1]; bb++)
            c_next[k].push_back({p.T.sons[a], p.S.sons[bb]});
      }
    });
    std::vector<std::pair<int32_t, int32_t>> fpairs, next;
    for (int k = 0; k < K; k++) {
      fpairs.insert(fpairs.end(), c_far[k].begin(), c_far[k].end());
      std::vector<std::pair<int32_t, int32_t>>().swap(c_far[k]);
      near_pairs.insert(near_pairs.end(), c_near[k].begin(), c_near[k].end());
      std::vector<std::pair<int32_t, int32_t>>().swap(c_near[k]);
      next.insert(next.end(), c_next[k].begin(), c_next[k].end());
      std::vector<std::pair<int32_t, int32_t>>().swap(c_next[k]);
    }
    frontier.swap(next);
    std::vector<std::pair<int32_t, int32_t>>().swap(next);
    const int64_t nf = (int64_t)fpairs.size();
    if (hf) p.n_far_hf += nf; else p.n_far_lf += nf;

    // 2. fundamental index, hash and (for HF) the cone of each far pair.
    // The cone of a translation is the one chosen for its first pair in the
    // reference's depth-first order (M2L.hpp:189-197): first occurrence in
    // fpairs, which is in that order.
    int m = 0;
    for (int64_t i = 0; i < nf; i++)
      for (int k = 0; k < 3; k++)
        m = std::max(m, std::abs(p.T.idx[3 * fpairs[i].first + k] - p.S.idx[3 * fpairs[i].second + k]));
    const int64_t w = 2 * m + 1;
    auto zkey = [&](int64_t i) {
      const int32_t t = fpairs[i].first, s = fpairs[i].second;
      int64_t key = 0;
      for (int k = 0; k < 3; k++) key = key * w + (p.T.idx[3 * t + k] - p.S.idx[3 * s + k] + m);
      return key;
    };
    std::vector<int16_t> cone(hf ? nf : 0, -1);
    if (hf && nf) {
      std::vector<std::atomic<int64_t>> firstpos(w * w * w);
      for (auto& a : firstpos) a.store(INT64_MAX, std::memory_order_relaxed);
      pfor(nf, 4096, [&](int64_t i) {
        auto& a = firstpos[zkey(i)];
        int64_t cur = a.load(std::memory_order_relaxed);
        while (i < cur && !a.compare_exchange_weak(cur, i, std::memory_order_relaxed)) {
        }
      });
      std::vector<int64_t> firsts;
      for (int64_t k = 0; k < w * w * w; k++) {
        int64_t f = firstpos[k].load(std::memory_order_relaxed);
        if (f != INT64_MAX) firsts.push_back(f);
      }
      std::vector<int16_t> key_cone(w * w * w, -1);
      const auto& tab = p.dirs[v.HFStage[l]];
      pfor((int64_t)firsts.size(), 16, [&](int64_t j) {
        const int64_t i = firsts[j];
        const int32_t t = fpairs[i].first, s = fpairs[i].second;
        double fZ[3] = {p.T.ctr[3 * t] - p.S.ctr[3 * s], p.T.ctr[3 * t + 1] - p.S.ctr[3 * s + 1],
                        p.T.ctr[3 * t + 2] - p.S.ctr[3 * s + 2]};
        const double n = norm3(fZ);
        for (int k = 0; k < 3; k++) fZ[k] /= n;
        key_cone[zkey(i)] = (int16_t)nearest_direction(tab, fZ);
      });
      pfor(nf, 4096, [&](int64_t i) { cone[i] = key_cone[zkey(i)]; });
    }

    // 3. effective directions of this level (BlankHorizontalPass flags plus
    // the BlankDownwardPass propagation from the parent level,
    // dwnpass.hpp:81-109)
    LevelFlags fT, fS;
    fT.cells = lcT[l];
    fS.cells = lcS[l];
    const int nd = v.nDir[l];
    const bool hfprec = v.prec[l] && v.isHF[l];
    if (hfprec) {
      fT.eff.assign(fT.cells.size() * (size_t)nd, 0);
      fS.eff.assign(fS.cells.size() * (size_t)nd, 0);
      if (hf)
        pfor(nf, 4096, [&](int64_t i) {
          const int c = cone[i];
          __atomic_store_n(&fT.eff[(size_t)locT[fpairs[i].first] * nd + c], (uint8_t)1, __ATOMIC_RELAXED);
          __atomic_store_n(&fS.eff[(size_t)locS[fpairs[i].second] * nd + c], (uint8_t)1, __ATOMIC_RELAXED);
        });
      if (!v.noHF && l > 0 && v.isHF[l - 1] && v.prec[l - 1]) {
        const int pnd = v.nDir[l - 1];
        auto prop = [&](const Tree& tr, LevelFlags& cur, const LevelFlags& prev,
                        const std::vector<int32_t>& loc) {
          pfor((int64_t)cur.cells.size(), 256, [&](int64_t i) {
            const int64_t par = tr.parent[cur.cells[i]];
            const uint8_t* pe = &prev.eff[(size_t)loc[par] * pnd];
            uint8_t* ce = &cur.eff[(size_t)i * nd];
            for (int dt = 0; dt < nd; dt++)
              if (pe[4 * dt] | pe[4 * dt + 1] | pe[4 * dt + 2] | pe[4 * dt + 3]) ce[dt] = 1;
          });
        };
        prop(p.T, fT, fT_prev, locT);
        prop(p.S, fS, fS_prev, locS);
      }
    }

    // 4. slots of this level
    p.sT.lvl_begin[l] = p.sT.n;
    p.sS.lvl_begin[l] = p.sS.n;
    level_slots(p, l, fT, p.sT, denseT);
    level_slots(p, l, fS, p.sS, denseS);

    // 5. transfer-spectrum ids per fundamental index and the M2L entries
    if (nf) {
      std::vector<int32_t> tid((m + 1) * (m + 1) * (m + 1), -1);
      std::vector<uint8_t> hs(nf);
      std::vector<int32_t> fi(nf);
      pfor(nf, 4096, [&](int64_t i) {
        const int32_t t = fpairs[i].first, s = fpairs[i].second;
        int iZ[3], nI[3], h;
        for (int k = 0; k < 3; k++) iZ[k] = p.T.idx[3 * t + k] - p.S.idx[3 * s + k];
        symmetry(iZ, nI, h);
        hs[i] = (uint8_t)h;
        fi[i] = (nI[0] * (m + 1) + nI[1]) * (m + 1) + nI[2];
        __atomic_store_n(&tid[fi[i]], 0, __ATOMIC_RELAXED);
      });
      for (size_t k = 0; k < tid.size(); k++)
        if (tid[k] == 0) {
          tid[k] = (int32_t)table_count++;
          const int a = (int)(k / ((m + 1) * (m + 1))), b = (int)((k / (m + 1)) % (m + 1)),
                    c = (int)(k % (m + 1));
          tab_nI.push_back({a, b, c});
          p.tab_lvl.push_back(l);
          const int M = v.nCellMax[l];
          p.tab_iz.push_back(((int64_t)a * M + b) * M + c);
        }
      auto& fts = walk.far_ts[l];
      auto& fss = walk.far_ss[l];
      auto& ftab = walk.far_tab[l];
      fts.resize(nf);
      fss.resize(nf);
      ftab.resize(nf);
      pfor(nf, 4096, [&](int64_t i) {
        const int64_t lt = locT[fpairs[i].first], ls = locS[fpairs[i].second];
        const int32_t ts = hf ? denseT[lt * nd + cone[i]] : denseT[lt];
        const int32_t ss = hf ? denseS[ls * nd + cone[i]] : denseS[ls];
        fts[i] = ts;
        fss[i] = ss;
        ftab[i] = ((uint32_t)tid[fi[i]] << 6) | hs[i];
      });
      if (p.keep_lists) {
        for (int64_t i = 0; i < nf; i++) {
          const int32_t t = fpairs[i].first, s = fpairs[i].second;
          int iZ[3], nI[3], h;
          for (int k = 0; k < 3; k++) iZ[k] = p.T.idx[3 * t + k] - p.S.idx[3 * s + k];
          symmetry(iZ, nI, h);
          const int M = v.nCellMax[l];
          const int32_t iz = (int32_t)(((int64_t)nI[0] * M + nI[1]) * M + nI[2]);
          if (hf) {
            const int32_t r[6] = {t, s, l, cone[i], iz, h};
            p.rec_far_hf.insert(p.rec_far_hf.end(), r, r + 6);
          } else {
            const int32_t r[5] = {t, s, l, iz, h};
            p.rec_far_lf.insert(p.rec_far_lf.end(), r, r + 5);
          }
        }
      }
    }

    // 6. slot children (M2M) of the previous level and slot parents (L2L)
    // of this level now that both levels have their slots
    // (upwpass.hpp:37-64, dwnpass.hpp:37-62)
    fT_prev = std::move(fT);
    fS_prev = std::move(fS);
    denseT_prev.swap(denseT);
    denseS_prev.swap(denseS);
  }
  p.sT.lvl_begin[nlvl] = p.sT.n;
  p.sS.lvl_begin[nlvl] = p.sS.n;
  return 0;
}

int build_plan(Plan& p, const double* src, int64_t ns, const double* trg,
               int64_t nt, int L, int ncrit, double kappa, int lvmax,
               std::string& err, LevelWalker* walker, TreeSorter* sorter) {
  if (ns <= 0 || nt <= 0) {
    err = "empty source or target set";
    return -1;
  }
  if (L < 2 || L > 8) {
    err = "interpolation order must be in [2, 8]";
    return -1;
  }
  if (lvmax < 0 && ncrit < 1) {
    err = "leaf size must be positive";
    return -1;
  }
  if (ns >= (int64_t(1) << 31) || nt >= (int64_t(1) << 31)) {
    err = "too many particles";
    return -1;
  }
  p.L = L;
  p.P = 2 * L - 1;
  p.LL = L * L * L;
  p.PP = p.P * p.P * p.P;
  p.ncrit = ncrit;
  p.lvmax = lvmax;
  p.kappa = kappa;
  p.p2p_sym = ns == nt && (src == trg || std::memcmp(src, trg, sizeof(double) * 3 * (size_t)ns) == 0);
  p.t_steps.clear();
  double t0 = now_s();
  // particles.hpp:79-100 (getBounds): one cube around targets and sources
  {
    double mn[3], mx[3];
    for (int k = 0; k < 3; k++) mn[k] = mx[k] = trg[k];
    auto upd = [&](const double* x, int64_t n) {
      for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
          const double a = x[3 * i + k];
          mn[k] = mn[k] < a ? mn[k] : a;
          mx[k] = mx[k] > a ? mx[k] : a;
        }
    };
    upd(trg, nt);
    upd(src, ns);
    for (int k = 0; k < 3; k++) p.box_ctr[k] = (mn[k] + mx[k]) / 2.;
    double a = p.box_ctr[0] - mn[0], b = mx[0] - p.box_ctr[0];
    for (int k = 1; k < 3; k++) {
      a = a > p.box_ctr[k] - mn[k] ? a : p.box_ctr[k] - mn[k];
      b = b > mx[k] - p.box_ctr[k] ? b : mx[k] - p.box_ctr[k];
    }
    p.box_rad = std::max(a, b);
  }
  int st = build_tree(p.T, trg, nt, p.box_ctr, p.box_rad, ncrit, lvmax, err, sorter);
  if (st) return st;
  st = build_tree(p.S, src, ns, p.box_ctr, p.box_rad, ncrit, lvmax, err, sorter);
  if (st) return st;
  p.tree_on_device = sorter != nullptr;
  p.t_tree = now_s() - t0;
  p.t_steps.push_back({"octrees (bounds, particle ordering, cells)", p.t_tree});
  t0 = now_s();
  double ts = t0;
  st = init_levels(p, err);
  if (st) return st;
  init_directions(p);
  init_small_tables(p);
  const bool dev_tables = walker && !p.keep_lists;
  p.tables_on_device = dev_tables;
  init_signatures(p, !dev_tables);
  p.step("levels, directions, small tables, signatures", ts);
  const Levels& v = p.lv;
  const int nlvl = v.nlvl;

  LevelWalk w;
  const double tw = now_s();
  st = (walker && !p.keep_lists) ? walker->walk(p, w, err) : walk_levels_host(p, w);
  if (st) return st;
  p.t_walk = now_s() - tw;
  if (!walker || p.keep_lists) p.t_steps.push_back({"level walk (host)", p.t_walk});
  ts = now_s();
  auto& near_pairs = w.near_pairs;
  auto& tab_nI = w.tab_nI;

  // per-cell direction/slot CSR for both trees
  auto cell_csr = [&](const Tree& tr, Slots& s) {
    s.cell_dirs.resize(s.n);
    s.cell_slots.resize(s.n);
    // slots of one cell appear in increasing direction order (cone-major)
    bucket_sort(s.n, tr.ncell, s.cell_ptr, [&](int64_t k) { return (int64_t)s.cell[k]; },
                [&](int64_t pos, int64_t k) {
                  s.cell_dirs[pos] = s.dir[k];
                  s.cell_slots[pos] = k;
                });
  };
  if (!w.cells_done) {
    cell_csr(p.T, p.sT);
    cell_csr(p.S, p.sS);
    p.step("slots per cell", ts);
  }

  // M2L grouped by target slot, each slot's entries by increasing source
  // slot (so that consecutive target slots can be merged on their common
  // sources; a slot meets each source slot at most once)
  if (!w.m2l_done) {
    p.m2l_ptr.assign(p.sT.n + 1, 0);
    for (int l = 0; l < nlvl; l++)
      for (int32_t ts : w.far_ts[l]) p.m2l_ptr[ts + 1]++;
    for (int64_t k = 0; k < p.sT.n; k++) p.m2l_ptr[k + 1] += p.m2l_ptr[k];
    const int64_t tot = p.m2l_ptr[p.sT.n];
    p.m2l_src.resize(tot);
    p.m2l_tab.resize(tot);
    std::vector<int64_t> pos(p.m2l_ptr.begin(), p.m2l_ptr.end() - 1);
    for (int l = 0; l < nlvl; l++) {
      for (size_t i = 0; i < w.far_ts[l].size(); i++) {
        const int64_t q = pos[w.far_ts[l][i]]++;
        p.m2l_src[q] = w.far_ss[l][i];
        p.m2l_tab[q] = w.far_tab[l][i];
      }
      std::vector<int32_t>().swap(w.far_ts[l]);
      std::vector<int32_t>().swap(w.far_ss[l]);
      std::vector<uint32_t>().swap(w.far_tab[l]);
    }
    pfor(p.sT.n, 1024, [&](int64_t t) {  // insertion sort: a slot has a few hundred entries at most
      const int64_t b = p.m2l_ptr[t], e = p.m2l_ptr[t + 1];
      for (int64_t q = b + 1; q < e; q++) {
        const int32_t sq = p.m2l_src[q];
        const uint32_t kq = p.m2l_tab[q];
        int64_t r = q;
        for (; r > b && p.m2l_src[r - 1] > sq; r--) {
          p.m2l_src[r] = p.m2l_src[r - 1];
          p.m2l_tab[r] = p.m2l_tab[r - 1];
        }
        p.m2l_src[r] = sq;
        p.m2l_tab[r] = kq;
      }
    });
  }

  // permuted spectra: one per (spectrum, symmetry hash) pair that occurs
  if (!w.m2l_done) {
    const int64_t ntab = (int64_t)tab_nI.size();
    std::vector<int32_t> pid(ntab * 64, -1);
    for (uint32_t k : p.m2l_tab) pid[k] = 0;
    p.ptab_key.clear();
    for (int64_t k = 0; k < ntab * 64; k++)
      if (pid[k] == 0) {
        pid[k] = (int32_t)p.ptab_key.size();
        p.ptab_key.push_back((uint32_t)k);
      }
    pfor((int64_t)p.m2l_tab.size(), 1 << 16, [&](int64_t e) { p.m2l_tab[e] = (uint32_t)pid[p.m2l_tab[e]]; });
  }

  p.step("M2L entries by target slot, permuted spectra", ts);
  // CSR over slots from a per-slot visitor visit(k, emit), in slot order:
  // blocks of slots are visited in parallel once, each into its own buffer
  // (ptr holding block-local offsets), then shifted and copied into place
  auto slot_csr = [&](int64_t n, auto visit, std::vector<int64_t>& ptr, std::vector<int32_t>& out) {
    constexpr int64_t B = 1 << 15;  // slots per block
    const int64_t nb = (n + B - 1) / B;
    std::vector<std::vector<int32_t>> part(nb);
    ptr.assign(n + 1, 0);
    pfor(nb, 1, [&](int64_t b) {
      const int64_t k1 = std::min(n, (b + 1) * B);
      auto& v = part[b];
      for (int64_t k = b * B; k < k1; k++) {
        visit(k, [&](int64_t x) { v.push_back((int32_t)x); });
        ptr[k + 1] = (int64_t)v.size();
      }
    });
    std::vector<int64_t> boff(nb + 1, 0);
    for (int64_t b = 0; b < nb; b++) boff[b + 1] = boff[b] + (int64_t)part[b].size();
    out.resize(boff[nb]);
    pfor(nb, 1, [&](int64_t b) {
      const int64_t k1 = std::min(n, (b + 1) * B);
      for (int64_t k = b * B; k < k1; k++) ptr[k + 1] += boff[b];
      std::copy(part[b].begin(), part[b].end(), out.begin() + boff[b]);
      std::vector<int32_t>().swap(part[b]);
    });
  };
  // M2M: children slots of each source slot (P2M/M2M operators, M2M.hpp:35-124)
  if (!w.transfers_done) {
    const Slots& s = p.sS;
    slot_csr(
        s.n,
        [&](int64_t k, auto emit) {
          const int64_t c = s.cell[k];
          const int l = p.S.lvl[c];
          if (!v.prec[l] || p.S.leaf(c)) return;
          const int d = s.dir[k];
          const bool hfd = v.isHF[l] && v.HFStage[l] > 0;
          for (int64_t a = p.S.son_ptr[c]; a < p.S.son_ptr[c + 1]; a++) {
            const int64_t cs = s.slot_of(p.S.sons[a], hfd ? d / 4 : -1);
            if (cs >= 0) emit(cs);
          }
        },
        p.m2m_ptr, p.m2m_child);
  }
  // L2L: parent slots feeding each target slot (L2L.hpp:35-127)
  if (!w.transfers_done) {
    const Slots& s = p.sT;
    slot_csr(
        s.n,
        [&](int64_t k, auto emit) {
          const int64_t c = s.cell[k];
          const int64_t pc = p.T.parent[c];
          if (pc < 0) return;
          const int l = p.T.lvl[pc];
          if (!v.prec[l]) return;
          const int dt = s.dir[k];
          const int64_t b = s.cell_ptr[pc], e = s.cell_ptr[pc + 1];
          if (v.isHF[l] && v.HFStage[l] > 0) {  // parent directions 4dt..4dt+3
            // cell_dirs of the parent are increasing: binary search the run
            const int32_t* cd = s.cell_dirs.data();
            int64_t j = std::lower_bound(cd + b, cd + e, 4 * dt) - cd;
            for (; j < e && cd[j] / 4 == dt; j++) emit(s.cell_slots[j]);
          } else {  // HFStage-0 parent: all its directions; LF parent: its expansion
            for (int64_t j = b; j < e; j++) emit(s.cell_slots[j]);
          }
        },
        p.l2l_ptr, p.l2l_parent);
  }
  p.step("M2M and L2L transfer lists", ts);
  // leaves holding expansions (upwpass.hpp:39-47, dwnpass.hpp:39-47)
  for (int64_t c = 0; c < p.S.ncell; c++)
    if (p.S.leaf(c) && v.prec[p.S.lvl[c]]) p.p2m_leaf.push_back((int32_t)c);
  for (int64_t c = 0; c < p.T.ncell; c++)
    if (p.T.leaf(c) && v.prec[p.T.lvl[c]]) p.l2p_leaf.push_back((int32_t)c);

  // near field per target leaf: a near pair (t, s) sends the particles of s
  // to every particle below t (P2P.hpp:43-79 on whole subtrees); the device
  // walk may have built these lists already (Plan::nd)
  if (!w.near_done) {
    p.n_near = (int64_t)near_pairs.size();
    if (p.keep_lists)
      for (auto& pr : near_pairs) {
        p.rec_near.push_back(pr.first);
        p.rec_near.push_back(pr.second);
      }
    // source ranges per target leaf, in pair order: K contiguous blocks of
    // pairs count per leaf, then fill after the blocks before them
    const int64_t npair = (int64_t)near_pairs.size();
    const int K = (int)std::max<int64_t>(1, std::min<int64_t>(std::min<unsigned>(hw_threads(), 32), npair / 4096 + 1));
    std::vector<std::vector<int64_t>> kc(K, std::vector<int64_t>(p.T.ncell, 0));
    std::vector<int64_t> kin(K, 0);
    pchunks(npair, K, [&](int k, int64_t b, int64_t e) {
      for (int64_t i = b; i < e; i++) {
        const auto& pr = near_pairs[i];
        for (int64_t c = pr.first; c < p.T.sub_end[pr.first]; c++)
          if (p.T.leaf(c)) kc[k][c]++;
        kin[k] += (int64_t)p.T.nprt[pr.first] * p.S.nprt[pr.second];
      }
    });
    std::vector<int64_t> cnt(p.T.ncell + 1, 0);
    for (int64_t c = 0; c < p.T.ncell; c++) {
      int64_t n = cnt[c];
      for (int k = 0; k < K; k++) {
        const int64_t v = kc[k][c];
        kc[k][c] = n;
        n += v;
      }
      cnt[c + 1] = n;
    }
    for (int k = 0; k < K; k++) p.i_near += kin[k];
    std::vector<std::pair<int32_t, int32_t>> rng(cnt[p.T.ncell]);
    pchunks(npair, K, [&](int k, int64_t b, int64_t e) {
      for (int64_t i = b; i < e; i++) {
        const auto& pr = near_pairs[i];
        const int32_t sf = p.S.first[pr.second], sn = p.S.nprt[pr.second];
        for (int64_t c = pr.first; c < p.T.sub_end[pr.first]; c++)
          if (p.T.leaf(c)) rng[kc[k][c]++] = {sf, sn};
      }
    });
    std::vector<std::vector<int64_t>>().swap(kc);
    std::vector<std::pair<int32_t, int32_t>>().swap(near_pairs);
    // merge touching ranges per leaf
    std::vector<std::vector<std::pair<int32_t, int32_t>>> merged(p.T.ncell);
    pfor(p.T.ncell, 256, [&](int64_t c) {
      if (cnt[c] == cnt[c + 1]) return;
      std::vector<std::pair<int32_t, int32_t>> r(rng.begin() + cnt[c], rng.begin() + cnt[c + 1]);
      std::sort(r.begin(), r.end());
      auto& out = merged[c];
      for (auto& x : r) {
        if (!out.empty() && out.back().first + out.back().second == x.first)
          out.back().second += x.second;
        else
          out.push_back(x);
      }
    });
    // chunks of <= 32 targets per leaf, each with the leaf's ranges: offsets
    // per leaf in leaf order, then a parallel fill
    std::vector<int64_t> ch_off(p.T.ncell + 1, 0), rg_off(p.T.ncell + 1, 0);
    for (int64_t c = 0; c < p.T.ncell; c++) {
      const int64_t nch = merged[c].empty() ? 0 : (p.T.nprt[c] + 31) / 32;
      ch_off[c + 1] = ch_off[c] + nch;
      rg_off[c + 1] = rg_off[c] + nch * (int64_t)merged[c].size();
    }
    p.p2p_tfirst.resize(ch_off[p.T.ncell]);
    p.p2p_tn.resize(ch_off[p.T.ncell]);
    p.p2p_ptr.assign(ch_off[p.T.ncell] + 1, 0);
    p.p2p_sfirst.resize(rg_off[p.T.ncell]);
    p.p2p_sn.resize(rg_off[p.T.ncell]);
    pfor(p.T.ncell, 64, [&](int64_t c) {
      if (merged[c].empty()) return;
      int64_t q = ch_off[c], r = rg_off[c];
      for (int32_t off = 0; off < p.T.nprt[c]; off += 32, q++) {
        p.p2p_tfirst[q] = p.T.first[c] + off;
        p.p2p_tn[q] = std::min(32, p.T.nprt[c] - off);
        for (auto& x : merged[c]) {
          p.p2p_sfirst[r] = x.first;
          p.p2p_sn[r] = x.second;
          r++;
        }
        p.p2p_ptr[q + 1] = r;
      }
    });
    p.step("near-field ranges and chunks", ts);
    if (p.p2p_sym) {
      build_symmetric_near(p);
      split_items(p, p.sym_ptr, p.sym_sfirst, p.sym_sn, &p.sym_soff, p.sym_item_chunk, p.sym_chunk_items,
                  p.sym_order, true);
    }
    split_items(p, p.p2p_ptr, p.p2p_sfirst, p.p2p_sn, nullptr, p.p2p_item_chunk, p.p2p_chunk_items, p.p2p_order,
                false);
    p.step("near-field symmetric blocks and work items", ts);
  }
  p.t_lists = now_s() - t0;

  // transfer spectra, FP64 (circulant.hpp:133-144); with a device plan the
  // device computes them (and the signatures) when the operator uploads
  t0 = now_s();
  const int64_t ntab = (int64_t)tab_nI.size();
  p.tables.clear();
  p.tab_fund.clear();
  if (dev_tables) {
    p.tab_fund = std::move(tab_nI);
  } else {
    p.tables.assign(ntab * (size_t)p.PP, cplx(0., 0.));
    pfor(ntab, 8, [&](int64_t k) {
      const int l = p.tab_lvl[k];
      const double rad = p.box_rad / (double)(1 << l);
      transfer_spectrum(p, rad, tab_nI[k].data(), &p.tables[k * (size_t)p.PP]);
    });
  }
  p.t_tables = now_s() - t0;
  p.step(dev_tables ? "transfer spectra (left to the device)" : "transfer spectra (FP64)", ts);
  return 0;
}

}  // namespace dfb
