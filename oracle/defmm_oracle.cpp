// =============================================================================
// ORACLE -- test infrastructure only.  Never linked into, loaded by or called
// from the product path; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg may use it, and only as the checker.
//
// A plain C++ restatement of the reference defmm's directional equispaced-
// interpolation FMM for the Helmholtz kernel exp(i k r)/(4 pi r) in 3-D
// (IChollet/defmm, include/interface.hpp:100-170), written from the
// reference's semantics, one function per reference step, each citing the
// reference file:line it follows.  It is pinned against the reference itself
// (oracle/_ref/defmm_ref, the unmodified reference built by oracle/Makefile):
// bit-exact trees, cones and interaction lists, potentials to rounding.
//
// Arithmetic follows the reference's operation order where the result is
// compared bit-exactly (tree centres, admissibility, cones); elsewhere FP64
// rounding may differ from the reference at the 1e-15 level.
//
// Deliberate difference: every gemv starts from zeroed expansions (the
// reference zeroes only the potentials, interface.hpp:159, so only its first
// gemv after prcmpt is valid).
// =============================================================================
#include <algorithm>
#include <atomic>
#include <mutex>
#include <thread>
#include <array>
#include <tuple>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

namespace {

typedef std::complex<double> cplx;

// Minimal parallel loop over [0, n) in dynamic chunks (std::thread; the
// oracle is built without an OpenMP runtime).
template <typename F>
void parallel_for(long n, long chunk, F f) {
  unsigned nt = std::max(1u, std::thread::hardware_concurrency());
  std::atomic<long> next(0);
  auto work = [&]() {
    for (;;) {
      long b = next.fetch_add(chunk);
      if (b >= n) return;
      long e = std::min(n, b + chunk);
      for (long i = b; i < e; i++) f(i);
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; t++) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}
const double kPi4 = 4. * M_PI;

// ---------------------------------------------------------------- geometry --
struct Particle {
  double pos[3];
  int ind;  // user index (tree.hpp:66-70)
};

struct Cell {
  int idx[3];
  int lvl;
  int nprt;
  double ctr[3];
  double rad;
  int first;  // first particle (tree order), sort.hpp:177
  std::vector<int> son;
  // directional data
  std::vector<int> slot;  // effDir: 0 = unused, else 1-based slot (initdevs.hpp:196)
  std::vector<int> dirs;  // effective directions, increasing
  int nexp = 0;           // number of expansions held by this cell
  long exp0 = -1;         // first expansion slot in the per-tree arrays
  // leaf data
  std::vector<double> zmat;             // LL x n (source) or n x LL (target)
  std::vector<std::vector<cplx>> sigs;  // per effective dir, n values
};

struct Tree {
  std::vector<Particle> parts;
  std::vector<Cell> cells;
  int nlvl = 0;
};

// particles.hpp:79-100 (getBounds): shared cube over both sets
void get_bounds(const std::vector<Particle>& t, const std::vector<Particle>& s,
                double ctr[3], double& rad) {
  double mn[3], mx[3];
  for (int k = 0; k < 3; k++) mn[k] = mx[k] = t[0].pos[k];
  for (size_t i = 1; i < t.size(); i++)
    for (int k = 0; k < 3; k++) {
      mn[k] = mn[k] < t[i].pos[k] ? mn[k] : t[i].pos[k];
      mx[k] = mx[k] > t[i].pos[k] ? mx[k] : t[i].pos[k];
    }
  for (size_t i = 0; i < s.size(); i++)
    for (int k = 0; k < 3; k++) {
      mn[k] = mn[k] < s[i].pos[k] ? mn[k] : s[i].pos[k];
      mx[k] = mx[k] > s[i].pos[k] ? mx[k] : s[i].pos[k];
    }
  for (int k = 0; k < 3; k++) ctr[k] = (mn[k] + mx[k]) / 2.;
  double a = ctr[0] - mn[0], b = mx[0] - ctr[0];
  for (int k = 1; k < 3; k++) {
    a = a > ctr[k] - mn[k] ? a : ctr[k] - mn[k];
    b = b > mx[k] - ctr[k] ? b : mx[k] - ctr[k];
  }
  rad = std::max(a, b);
}

// sort.hpp:98-162 (rcSort) + sort.hpp:187-220 (rcCreateCells): recursive
// stable 8-way bucket split on (pos[k] > ctr[k]) << k; a cell is a leaf when
// it holds fewer than ncrit particles (sort.hpp:49), or, with lvmax >= 0,
// when lvl >= lvmax (sort.hpp:51).  Cells are emitted in DFS pre-order.
struct Builder {
  std::vector<Particle>* parts;
  std::vector<Cell>* cells;
  int ncrit, lvmax;
  int maxlvl = 0;
  bool overflow = false;

  bool stop(int n, int lvl) const {
    return lvmax >= 0 ? lvl >= lvmax : n < ncrit;
  }

  void build(int first, int n, const double ctr[3], double rad,
             const int idx[3], int lvl) {
    int me = (int)cells->size();
    cells->push_back(Cell());
    Cell& c = (*cells)[me];
    for (int k = 0; k < 3; k++) {
      c.idx[k] = idx[k];
      c.ctr[k] = ctr[k];
    }
    c.lvl = lvl;
    c.nprt = n;
    c.rad = rad;
    c.first = first;
    maxlvl = std::max(maxlvl, lvl);
    if (stop(n, lvl)) return;
    if (lvl >= 60) {  // coincident points: the reference recurses forever
      overflow = true;
      return;
    }
    std::vector<Particle> tmp(parts->begin() + first,
                              parts->begin() + first + n);
    int histo[8] = {0}, off[8], add[8] = {0};
    std::vector<int> code(n);
    for (int i = 0; i < n; i++) {
      int b = 0;
      for (int k = 0; k < 3; k++) b += ((tmp[i].pos[k] > ctr[k]) ? 1 : 0) << k;
      code[i] = b;
      histo[b]++;
    }
    off[0] = 0;
    for (int i = 1; i < 8; i++) off[i] = off[i - 1] + histo[i - 1];
    for (int i = 0; i < n; i++)
      (*parts)[first + off[code[i]] + add[code[i]]++] = tmp[i];
    double nrad = rad / 2.;
    for (int b = 0; b < 8; b++) {
      if (!histo[b]) continue;
      double nc[3];
      int ni[3];
      for (int k = 0; k < 3; k++) {
        nc[k] = ctr[k] + nrad * (double)(((b >> k) & 1) * 2 - 1);
        ni[k] = 2 * idx[k] + ((b >> k) & 1);
      }
      int child = (int)cells->size();
      (*cells)[me].son.push_back(child);
      build(first + off[b], histo[b], nc, nrad, ni, lvl + 1);
      if (overflow) return;
    }
  }
};

// ------------------------------------------------------------- directions --
// newdirections.hpp:76-171 (iterativeGetDirections)
struct Directions {
  std::vector<std::vector<std::array<double, 3>>> tab;
};

double norm3(const double* v) {
  double t = 0.;
  for (int i = 0; i < 3; i++) t += v[i] * v[i];
  return std::sqrt(t);
}

void get_directions(Directions& D, int nstages) {
  D.tab.assign(nstages, {});
  for (int e = 0; e < nstages; e++) D.tab[e].assign((size_t)6 << (2 * e), {0, 0, 0});
  if (nstages == 0) return;
  for (int k = 0; k < 3; k++) {
    D.tab[0][2 * k] = {0, 0, 0};
    D.tab[0][2 * k][k] = 1.;
    D.tab[0][2 * k + 1] = {0, 0, 0};
    D.tab[0][2 * k + 1][k] = -1.;
  }
  double hyp[4][3];
  for (int q = 0; q < 4; q++) {
    hyp[q][0] = 0.;
    hyp[q][1] = (q & 1) ? -1. : 1.;
    hyp[q][2] = (q & 2) ? -1. : 1.;
  }
  int npe = 1;
  for (int e = 1; e < nstages; e++) {
    double radius = 1. / (double)(1 << (e + 1));
    for (int i = 0; i < npe; i++)
      for (int q = 0; q < 4; q++) {
        auto d = D.tab[e - 1][i];
        for (int k = 0; k < 3; k++) d[k] += hyp[q][k] * radius;
        double nr = norm3(d.data());
        for (int k = 0; k < 3; k++) d[k] /= nr;
        D.tab[e][i * 4 + q] = d;
      }
    npe *= 4;
  }
  // reflection of the +x face onto the -x face (only block 1 survives the
  // rotation step below; newdirections.hpp:131-141)
  int fs = 1;
  for (int e = 1; e < nstages; e++) {
    fs *= 4;
    for (int j = 0; j < 4 * fs; j++) {
      auto d = D.tab[e][j];
      d[0] *= -1.;
      D.tab[e][fs + j] = d;
    }
  }
  // rotations (newdirections.hpp:144-155): block pair j gets d[k] = src[(k+j)%3]
  fs = 1;
  for (int e = 1; e < nstages; e++) {
    fs *= 4;
    int f2 = 2 * fs;
    for (int j = 1; j < 3; j++)
      for (int ii = 0; ii < f2; ii++)
        for (int k = 0; k < 3; k++) D.tab[e][j * f2 + ii][k] = D.tab[e][ii][(k + j) % 3];
  }
}

// newdirections.hpp:175-185: nearest direction, first index on ties
int best_cone(const Directions& D, int stage, const double* dir) {
  double tmp = 1.e30;
  int ind = -1;
  const auto& t = D.tab[stage];
  for (size_t i = 0; i < t.size(); i++) {
    double df[3] = {t[i][0] - dir[0], t[i][1] - dir[1], t[i][2] - dir[2]};
    double n = norm3(df);
    if (tmp > n) {
      tmp = n;
      ind = (int)i;
    }
  }
  return ind;
}

// -------------------------------------------------------------- symmetries --
// hypercube.hpp:109-136, permutations.hpp:88-120 and :128-150, :209-232
const int kSigma[8][3] = {{0, 1, 2}, {1, 0, 2}, {0, 1, 2}, {1, 2, 0},
                          {0, 2, 1}, {0, 1, 2}, {2, 0, 1}, {2, 1, 0}};

int hash_sigma(const int* I) {
  int h = 0, u = 0;
  for (int k = 0; k < 3; k++)
    for (int l = k + 1; l < 3; l++) h += ((std::abs(I[k]) < std::abs(I[l])) ? 1 : 0) << u++;
  return h;
}
int hash_sign(const int* I) {
  int h = 0;
  for (int k = 0; k < 3; k++) h += ((I[k] < 0) ? 1 : 0) << k;
  return h;
}
// fundamental multi-index nI and hash code p0 + (p1 << 3)
void fundamental(const int* iZ, int* nI, int& hsh) {
  int h1 = hash_sigma(iZ);
  for (int k = 0; k < 3; k++) nI[k] = std::abs(iZ[kSigma[h1][k]]);
  hsh = hash_sign(iZ) + (h1 << 3);
}

// ------------------------------------------------------ polynomials / keys --
// thetis_keys.hpp:35-53 (last index fastest); thetis_polynomials.hpp:81-94,126
inline void i2I(int i, int L, int* I) {
  for (int ii = 0; ii < 3; ii++) {
    I[2 - ii] = i % L;
    i -= I[2 - ii];
    i /= L;
  }
}
inline int I2i(const int* I, int L) { return (I[0] * L + I[1]) * L + I[2]; }
inline double point1D(int i, int L, double alpha) {
  return alpha * (-1. + 2. * ((double)i / (double)(L - 1)));
}
double S1D(int i, double x, int P, double alpha) {
  double res = 1., nx = x / alpha;
  double pi = -1. + 2. * ((double)i / (double)(P - 1));
  for (int ii = 0; ii < P; ii++) {
    if (ii == i) continue;
    double pii = -1. + 2. * ((double)ii / (double)(P - 1));
    res *= (nx - pii) / (pi - pii);
  }
  return res;
}

// -------------------------------------------------------------------- DFT --
// Direct 3-D DFT of size P (row-major), unnormalised; sign -1 forward.
struct Dft {
  int P;
  std::vector<cplx> wf, wb;
  void init(int p) {
    P = p;
    wf.resize(P);
    wb.resize(P);
    for (int m = 0; m < P; m++) {
      long double a = 2.0L * 3.14159265358979323846264338327950288L * m / P;
      wf[m] = cplx((double)cosl(a), -(double)sinl(a));
      wb[m] = std::conj(wf[m]);
    }
  }
  void run(cplx* x, bool fwd) const {
    const std::vector<cplx>& w = fwd ? wf : wb;
    cplx line[32], res[32];
    int inner = 1;
    for (int d = 2; d >= 0; d--) {
      int outer = P * P * P / (P * inner);
      for (int o = 0; o < outer; o++)
        for (int i = 0; i < inner; i++) {
          cplx* b = x + o * P * inner + i;
          for (int j = 0; j < P; j++) line[j] = b[j * inner];
          for (int k = 0; k < P; k++) {
            cplx acc = 0.;
            int m = 0;
            for (int j = 0; j < P; j++) {
              acc += line[j] * w[m];
              m += k;
              if (m >= P) m -= P;
            }
            res[k] = acc;
          }
          for (int k = 0; k < P; k++) b[k * inner] = res[k];
        }
      inner *= P;
    }
  }
};

// ------------------------------------------------------------------ state --
struct Oracle {
  int L, P, LL, PP, ncrit, lvmax;
  double kappa;
  double box_ctr[3], box_rad;
  Tree S, T;
  int nlvl = 0, cpt = 0, max_stage = 0;
  bool noHF = true;
  std::vector<int> isHF, HFStage, nDir, nCellMax;
  std::vector<char> prec;
  Directions D;
  std::vector<int> itilda;
  std::vector<double> tabZ;
  std::vector<std::vector<int>> perm;  // 64 x PP
  Dft dft;
  // transfer spectra: key (lvl, iz) -> table; dirTable: (lvl, iz, hsh) -> cone
  std::map<std::pair<int, long>, std::vector<cplx>> m2l;
  std::map<std::tuple<int, long, int>, int> cone;
  // signatures per level (HFStage indexing as planewave.hpp:44-69)
  std::map<int, std::vector<std::vector<cplx>>> sig, sig2;
  double m2m[2][64], l2l[2][64];  // real L x L, column-major
  // lists (HorizontalPass DFS order)
  std::vector<int32_t> near, far_hf, far_lf;
  int status = 0;
  // expansions (flattened)
  std::vector<cplx> Ms, Fs, Ls, Js;
  long nsrc_exp = 0, ntrg_exp = 0;
};

int n_levels(const Tree& t) {
  int m = 0;
  for (auto& c : t.cells) m = std::max(m, c.lvl);
  return m + 1;
}

// frequency.hpp:44-82 (fixFrequencyRegime), :90-98, :109-129, :159-184
int init_frequency(Oracle& o) {
  o.nlvl = std::max(n_levels(o.T), n_levels(o.S));
  double diam = 2. * o.box_rad;
  int cpt = 0;
  if (diam * o.kappa > 1.) {
    while (diam * o.kappa > 1.) {
      diam /= 2.;
      cpt++;
    }
  }
  o.cpt = cpt;
  if (cpt) get_directions(o.D, cpt);
  o.noHF = !(cpt > 1);
  o.isHF.assign(o.nlvl, 0);
  o.HFStage.assign(o.nlvl, 0);
  int hf = 1;
  for (int l = cpt; l > -1; l--) {
    if (l < o.nlvl) {
      o.isHF[l] = hf;
      o.HFStage[l] = hf - 1;
    }
    hf++;
  }
  o.nDir.assign(o.nlvl, 1);
  for (int l = o.nlvl - 1; l > -1; l--)
    if (o.isHF[l] && l != 0) o.nDir[l] = 6 << (2 * o.HFStage[l]);
  int ms = 0;
  double bd = 2. * o.box_rad;
  while (1. < o.kappa * bd / (double)(1 << ms) / (double)(1 << ms)) {
    ms++;
    if (ms >= o.nlvl) return -3;  // frequency.hpp:114-120: no precomputation level
  }
  ms = std::max(ms, 2);
  o.max_stage = ms;
  o.prec.assign(o.nlvl, 0);
  for (int l = ms; l < o.nlvl; l++) o.prec[l] = 1;
  o.nCellMax.assign(o.nlvl, -1);
  for (int l = 0; l < o.nlvl; l++) {
    if (!o.prec[l]) continue;
    if (o.isHF[l])
      o.nCellMax[l] = 1 << l;
    else
      o.nCellMax[l] = o.isHF[l - 1] ? 8 : 4;
  }
  return 0;
}

// circulant.hpp:47-93 (precomputeCirculant): itilda and tabZ
void init_circulant(Oracle& o) {
  o.itilda.resize(o.LL);
  for (int i = 0; i < o.LL; i++) {
    int I[3];
    i2I(i, o.L, I);
    o.itilda[i] = I2i(I, o.P);
  }
  o.tabZ.resize(3 * o.PP);
  for (int i = 0; i < o.PP; i++) {
    int E[3];
    i2I(i, o.P, E);
    for (int k = 0; k < 3; k++) {
      E[k] = E[k] < o.L ? E[k] : -(2 * o.L - 1 - E[k]);
      int Ip = E[k] > -1 ? E[k] : 0, Jn = E[k] > -1 ? 0 : -E[k];
      o.tabZ[3 * i + k] = point1D(Ip, o.L, 1.) - point1D(Jn, o.L, 1.);
    }
  }
  o.dft.init(o.P);
  // permutations.hpp:128-150 (computePermutations)
  o.perm.assign(64, std::vector<int>(o.PP));
  for (int p0 = 0; p0 < 8; p0++)
    for (int p1 = 0; p1 < 8; p1++) {
      int h = p0 + (p1 << 3);
      for (int p = 0; p < o.PP; p++) {
        int tp[3], tm[3];
        i2I(p, o.P, tp);
        for (int k = 0; k < 3; k++) {
          tm[k] = tp[kSigma[p1][k]];
          if ((p0 & (1 << kSigma[p1][k])) && tm[k]) tm[k] = o.P - tm[k];
        }
        o.perm[h][p] = I2i(tm, o.P);
      }
    }
}

// circulant.hpp:133-144 (fillCircCoeffs<3,Helmholtz>)
std::vector<cplx> transfer_spectrum(const Oracle& o, double rad, const double* v) {
  std::vector<cplx> in(o.PP);
  for (int i = 0; i < o.PP; i++) {
    double z[3];
    for (int k = 0; k < 3; k++) z[k] = v[k] + o.tabZ[3 * i + k] * rad;
    double R = norm3(z);
    double a = R * o.kappa;
    in[i] = cplx(std::cos(a), std::sin(a)) / (kPi4 * R);
  }
  o.dft.run(in.data(), true);
  return in;
}

// MAClist (hrzpass.hpp:40-49), MACgeomhf (hrzpass.hpp:52-56)
bool mac_list(const Cell& X, const Cell& Y) {
  int test = 0, ncmp = 3;
  for (int k = 0; k < 3; k++) {
    int d = X.idx[k] - Y.idx[k];
    ncmp -= d ? 0 : 1;
    test += std::abs(d);
  }
  return test > ncmp;
}
bool mac_hf(const Oracle& o, const Cell& X, const Cell& Y) {
  double d[3] = {X.ctr[0] - Y.ctr[0], X.ctr[1] - Y.ctr[1], X.ctr[2] - Y.ctr[2]};
  double tmp = (1. - 1.e-8) * (norm3(d) - 2. * Y.rad);
  double tt = 2. * Y.rad;
  return tmp >= std::max(tt * tt * o.kappa, tt);
}

long table_key(const Oracle& o, int lvl, const int* nI) {
  int m = o.nCellMax[lvl];
  return ((long)nI[0] * m + nI[1]) * m + nI[2];
}

// M2L.hpp:164-200 (blankM2Lhf): lazily create the HF spectrum, pick the cone
// of the first pair seen per (lvl, iz, hash), flag it on both cells.
void blank_m2l_hf(Oracle& o, Cell& t, Cell& s, std::vector<std::vector<char>>& teff,
                  std::vector<std::vector<char>>& seff, int ti, int si) {
  int iZ[3] = {t.idx[0] - s.idx[0], t.idx[1] - s.idx[1], t.idx[2] - s.idx[2]};
  int nI[3], hsh;
  fundamental(iZ, nI, hsh);
  long iz = table_key(o, t.lvl, nI);
  auto key = std::make_pair(t.lvl, iz);
  if (!o.m2l.count(key)) {
    double fV[3];
    for (int k = 0; k < 3; k++) fV[k] = 2. * (double)nI[k] * t.rad;
    o.m2l[key] = transfer_spectrum(o, t.rad, fV);
  }
  auto ck = std::make_tuple(t.lvl, iz, hsh);
  auto it = o.cone.find(ck);
  int c;
  if (it == o.cone.end()) {
    double fZ[3] = {t.ctr[0] - s.ctr[0], t.ctr[1] - s.ctr[1], t.ctr[2] - s.ctr[2]};
    double n = norm3(fZ);
    for (int k = 0; k < 3; k++) fZ[k] /= n;
    c = best_cone(o.D, o.HFStage[t.lvl], fZ);
    o.cone[ck] = c;
  } else {
    c = it->second;
  }
  teff[ti][c] = 1;
  seff[si][c] = 1;
}

// hrzpass.hpp:112-138 (BlankHorizontalPass)
void blank_hrz(Oracle& o, int i, int j, std::vector<std::vector<char>>& teff,
               std::vector<std::vector<char>>& seff) {
  Cell& X = o.T.cells[i];
  Cell& Y = o.S.cells[j];
  bool xhf = o.isHF[X.lvl], yhf = o.isHF[Y.lvl];
  if ((!xhf && !yhf) || (!xhf && Y.son.empty()) || (X.son.empty() && !yhf)) return;
  if (X.lvl == Y.lvl && mac_hf(o, X, Y) && o.prec[X.lvl]) {
    blank_m2l_hf(o, X, Y, teff, seff, i, j);
    return;
  }
  if (!X.son.empty() && !Y.son.empty())
    for (int a : X.son)
      for (int b : Y.son) blank_hrz(o, a, b, teff, seff);
}

// dwnpass.hpp:81-109 (BlankDownwardPass)
void blank_down(Oracle& o, Tree& tr, int c, std::vector<std::vector<char>>& eff) {
  Cell& C = tr.cells[c];
  if (C.son.empty()) return;
  if (o.isHF[C.lvl] && o.prec[C.lvl]) {
    for (int s : C.son) {
      if (C.lvl + 1 < o.nlvl && o.isHF[C.lvl + 1]) {
        for (int dt = 0; dt < o.nDir[C.lvl + 1]; dt++)
          for (int k = 0; k < 4; k++)
            if (eff[c][4 * dt + k]) eff[s][dt] = 1;
        blank_down(o, tr, s, eff);
      }
    }
  } else {
    for (int s : C.son) blank_down(o, tr, s, eff);
  }
}

// hrzpass.hpp:62-91 (HorizontalPass): enumerate far (M2L) and near (P2P)
// work in the reference's DFS order.
void hrz_lists(Oracle& o, int i, int j) {
  const Cell& X = o.T.cells[i];
  const Cell& Y = o.S.cells[j];
  if (o.prec[X.lvl] && X.lvl == Y.lvl) {
    if (X.lvl && o.isHF[X.lvl]) {
      if (mac_hf(o, X, Y)) {
        int iZ[3] = {X.idx[0] - Y.idx[0], X.idx[1] - Y.idx[1], X.idx[2] - Y.idx[2]};
        int nI[3], hsh;
        fundamental(iZ, nI, hsh);
        long iz = table_key(o, X.lvl, nI);
        int c = o.cone.at(std::make_tuple(X.lvl, iz, hsh));
        int32_t rec[6] = {i, j, X.lvl, c, (int32_t)iz, hsh};
        o.far_hf.insert(o.far_hf.end(), rec, rec + 6);
        return;
      }
    } else if (mac_list(X, Y)) {
      int iZ[3] = {X.idx[0] - Y.idx[0], X.idx[1] - Y.idx[1], X.idx[2] - Y.idx[2]};
      int nI[3], hsh;
      fundamental(iZ, nI, hsh);
      long iz = table_key(o, X.lvl, nI);
      int32_t rec[5] = {i, j, X.lvl, (int32_t)iz, hsh};
      o.far_lf.insert(o.far_lf.end(), rec, rec + 5);
      return;
    }
  }
  if (X.son.empty() || Y.son.empty()) {
    o.near.push_back(i);
    o.near.push_back(j);
    return;
  }
  for (int a : X.son)
    for (int b : Y.son) hrz_lists(o, a, b);
}

// initdevs.hpp:187-245 (InitializeDevs): compact 1-based slots
long assign_slots(Oracle& o, Tree& tr, std::vector<std::vector<char>>& eff) {
  long count = 0;
  for (size_t i = 0; i < tr.cells.size(); i++) {
    Cell& c = tr.cells[i];
    if (!o.prec[c.lvl]) continue;
    if (o.isHF[c.lvl]) {
      c.slot.assign(o.nDir[c.lvl], 0);
      int n = 0;
      for (int k = 0; k < o.nDir[c.lvl]; k++)
        if (eff[i][k]) {
          c.slot[k] = ++n;
          c.dirs.push_back(k);
        }
      c.nexp = n;
    } else {
      c.nexp = 1;
    }
    c.exp0 = count;
    count += c.nexp;
  }
  return count;
}

// planewave.hpp:44-69 (computeSignatures)
void init_signatures(Oracle& o) {
  for (int l = 2; l < o.nlvl; l++) {
    if (!(o.prec[l] && o.isHF[l])) continue;
    double locrad = o.box_rad / (double)(1 << l);
    int h = o.HFStage[l];
    auto& S1 = o.sig[h];
    auto& S2 = o.sig2[h];
    S1.assign(o.nDir[l], std::vector<cplx>(o.LL));
    S2.assign(o.nDir[l], std::vector<cplx>(o.LL));
    for (int i = 0; i < o.nDir[l]; i++) {
      const auto& d = o.D.tab[h][i];
      for (int k = 0; k < o.LL; k++) {
        int I[3];
        i2I(k, o.L, I);
        double x[3];
        for (int a = 0; a < 3; a++) x[a] = point1D(I[a], o.L, .5 * locrad);
        double dp = 0.;
        for (int a = 0; a < 3; a++) dp += d[a] * x[a];
        double ang = o.kappa * dp;
        S1[i][k] = cplx(std::cos(ang), -std::sin(ang));
        S2[i][k] = S1[i][k] * S1[i][k];
      }
    }
  }
}

// interpolation.hpp:184-242 (realPrecomputeM2M / realPrecomputeL2L)
void init_interp(Oracle& o) {
  for (int sg = 0; sg < 2; sg++)
    for (int p = 0; p < o.L; p++)
      for (int k = 0; k < o.L; k++) {
        double v = S1D(k, point1D(p, o.L, 1.) + (sg ? 1. : -1.), o.L, 2.);
        o.m2m[sg][k + p * o.L] = v;  // (k,p): parent basis k at child node p
        o.l2l[sg][p + k * o.L] = v;  // (p,k)
      }
}

// mapOnTrees.hpp:37-134 (fast{Source,Target}LeafMatrices)
void init_leaves(Oracle& o, Tree& tr, bool source) {
  for (auto& c : tr.cells) {
    if (!c.son.empty()) continue;
    int n = c.nprt;
    std::vector<double> Z(3 * o.L * n);
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < o.L; l++)
        for (int j = 0; j < n; j++)
          Z[(k * o.L + l) * n + j] =
              S1D(l, tr.parts[c.first + j].pos[k] - c.ctr[k], o.L, c.rad);
    c.zmat.assign((size_t)o.LL * n, 0.);
    for (int l = 0; l < o.LL; l++) {
      int I[3];
      i2I(l, o.L, I);
      for (int j = 0; j < n; j++) {
        double v = 1.;
        for (int k = 0; k < 3; k++) v *= Z[(k * o.L + I[k]) * n + j];
        if (source)
          c.zmat[l + (size_t)j * o.LL] = v;  // LL x n
        else
          c.zmat[j + (size_t)l * n] = v;  // n x LL
      }
    }
    if (o.isHF[c.lvl] && o.prec[c.lvl]) {
      for (int d : c.dirs) {
        const auto& dv = o.D.tab[o.HFStage[c.lvl]][d];
        std::vector<cplx> s(n);
        for (int j = 0; j < n; j++) {
          double df[3];
          for (int k = 0; k < 3; k++) df[k] = tr.parts[c.first + j].pos[k] - c.ctr[k];
          double dp = 0.;
          for (int k = 0; k < 3; k++) dp += dv[k] * df[k];
          double a = o.kappa * dp;
          s[j] = source ? cplx(std::cos(a), -std::sin(a)) : cplx(std::cos(a), std::sin(a));
        }
        c.sigs.push_back(s);
      }
    }
  }
}

// ------------------------------------------------------------- operators --
// separable 3-pass contraction (interpolation.hpp:311-361 / 463-513):
// out[a,b,c] = sum A_{s0}(a,a') A_{s1}(b,b') A_{s2}(c,c') in[a',b',c'],
// s_k = (v[k] < 0 ? 0 : 1); mats are column-major L x L, out(k) = sum_p m(k,p) in(p)
void separable(const Oracle& o, const double (*mats)[64], const double* v,
               const cplx* in, cplx* out) {
  const int L = o.L;
  std::vector<cplx> a(in, in + o.LL), b(o.LL);
  for (int it = 0; it < 3; it++) {
    int ax = 2 - it;
    const double* m = mats[v[ax] < 0. ? 0 : 1];
    for (int i = 0; i < o.LL; i++) {
      int I[3];
      i2I(i, L, I);
      cplx acc = 0.;
      for (int p = 0; p < L; p++) {
        int J[3] = {I[0], I[1], I[2]};
        J[ax] = p;
        acc += m[I[ax] + p * L] * a[I2i(J, L)];
      }
      b[i] = acc;
    }
    a.swap(b);
  }
  for (int i = 0; i < o.LL; i++) out[i] = a[i];
}

inline cplx expi(double a) { return cplx(std::cos(a), std::sin(a)); }
inline double dot3(const double* a, const double* b) {
  double r = 0.;
  for (int i = 0; i < 3; i++) r += a[i] * b[i];
  return r;
}

cplx* Mexp(Oracle& o, const Cell& c, int k) { return &o.Ms[(c.exp0 + k) * o.LL]; }
cplx* Fexp(Oracle& o, const Cell& c, int k) { return &o.Fs[(c.exp0 + k) * o.PP]; }
cplx* Lexp(Oracle& o, const Cell& c, int k) { return &o.Ls[(c.exp0 + k) * o.LL]; }
cplx* Jexp(Oracle& o, const Cell& c, int k) { return &o.Js[(c.exp0 + k) * o.PP]; }

// upwpass.hpp:37-64 with P2M.hpp:114-136 and M2M.hpp:35-124
void upward(Oracle& o, int ci, const cplx* q) {
  Cell& c = o.S.cells[ci];
  const int LL = o.LL;
  if (c.son.empty()) {
    if (!o.prec[c.lvl]) return;
    if (o.isHF[c.lvl]) {  // phfP2M
      const auto& s2 = o.sig2[o.HFStage[c.lvl]];
      for (int k = 0; k < c.nexp; k++) {
        cplx* M = Mexp(o, c, k);
        for (int l = 0; l < LL; l++) {
          cplx acc = 0.;
          for (int j = 0; j < c.nprt; j++)
            acc += c.zmat[l + (size_t)j * LL] * (c.sigs[k][j] * q[c.first + j]);
          M[l] = std::conj(s2[c.dirs[k]][l]) * acc;
        }
      }
    } else {  // plfP2M
      cplx* M = Mexp(o, c, 0);
      for (int l = 0; l < LL; l++) {
        cplx acc = 0.;
        for (int j = 0; j < c.nprt; j++) acc += c.zmat[l + (size_t)j * LL] * q[c.first + j];
        M[l] = acc;
      }
    }
    return;
  }
  for (int s : c.son) upward(o, s, q);
  if (!o.prec[c.lvl]) return;
  std::vector<cplx> buf(LL), res(LL);
  for (int si : c.son) {
    Cell& s = o.S.cells[si];
    double v[3] = {s.ctr[0] - c.ctr[0], s.ctr[1] - c.ctr[1], s.ctr[2] - c.ctr[2]};
    if (o.isHF[c.lvl]) {
      int h = o.HFStage[c.lvl];
      const auto& s1 = o.sig[h];
      const auto& s2 = o.sig2[h];
      for (int k = 0; k < c.nexp; k++) {
        int d = c.dirs[k];
        // hfM2Mblock uses the child's expansion of direction d/4; lf2hfM2M
        // (HFStage 0 parent) the child's single LF expansion
        const cplx* src = h ? Mexp(o, s, s.slot[d / 4] - 1) : Mexp(o, s, 0);
        for (int l = 0; l < LL; l++) buf[l] = s1[d][l] * src[l];
        separable(o, o.m2m, v, buf.data(), res.data());
        const auto& dv = o.D.tab[h][d];
        cplx edv = std::conj(expi(o.kappa * dot3(dv.data(), v)));
        cplx* M = Mexp(o, c, k);
        for (int l = 0; l < LL; l++) M[l] += std::conj(s2[d][l]) * res[l] * edv;
      }
    } else {  // lfM2M
      separable(o, o.m2m, v, Mexp(o, s, 0), res.data());
      cplx* M = Mexp(o, c, 0);
      for (int l = 0; l < LL; l++) M[l] += res[l];
    }
  }
}

// dwnpass.hpp:37-62 with L2L.hpp:35-127 and L2P.hpp:122-173
void downward(Oracle& o, int ci, cplx* p) {
  Cell& c = o.T.cells[ci];
  const int LL = o.LL;
  if (c.son.empty()) {
    if (!o.prec[c.lvl]) return;
    std::vector<cplx> buff(LL);
    if (o.isHF[c.lvl]) {  // phfL2P
      const auto& s2 = o.sig2[o.HFStage[c.lvl]];
      for (int k = 0; k < c.nexp; k++) {
        int d = c.dirs[k];
        const cplx* Lx = Lexp(o, c, k);
        for (int l = 0; l < LL; l++) buff[l] = s2[d][l] * Lx[l];
        const auto& dv = o.D.tab[o.HFStage[c.lvl]][d];
        for (int i = 0; i < c.nprt; i++) {
          cplx acc = 0.;
          for (int l = 0; l < LL; l++) acc += c.zmat[i + (size_t)l * c.nprt] * buff[l];
          double df[3];
          for (int a = 0; a < 3; a++) df[a] = o.T.parts[c.first + i].pos[a] - c.ctr[a];
          p[c.first + i] += acc * expi(o.kappa * dot3(dv.data(), df));
        }
      }
    } else {  // plfL2P
      const cplx* Lx = Lexp(o, c, 0);
      for (int i = 0; i < c.nprt; i++) {
        cplx acc = 0.;
        for (int l = 0; l < LL; l++) acc += c.zmat[i + (size_t)l * c.nprt] * Lx[l];
        p[c.first + i] += acc;
      }
    }
    return;
  }
  std::vector<cplx> buf(LL), res(LL);
  for (int ti : c.son) {
    Cell& t = o.T.cells[ti];
    if (o.prec[c.lvl]) {
      double v[3] = {t.ctr[0] - c.ctr[0], t.ctr[1] - c.ctr[1], t.ctr[2] - c.ctr[2]};
      if (o.isHF[c.lvl]) {
        int h = o.HFStage[c.lvl];
        const auto& s1 = o.sig[h];
        const auto& s2 = o.sig2[h];
        for (int k = 0; k < c.nexp; k++) {
          int d = c.dirs[k];
          const cplx* Lp = Lexp(o, c, k);
          for (int l = 0; l < LL; l++) buf[l] = s2[d][l] * Lp[l];
          separable(o, o.l2l, v, buf.data(), res.data());
          const auto& dv = o.D.tab[h][d];
          cplx ev = expi(o.kappa * dot3(v, dv.data()));
          // hfL2Lblock targets the child's direction d/4; hf2lfL2L (HFStage 0
          // parent) the child's single LF expansion
          cplx* Lc = h ? Lexp(o, t, t.slot[d / 4] - 1) : Lexp(o, t, 0);
          for (int l = 0; l < LL; l++) Lc[l] += std::conj(s1[d][l]) * res[l] * ev;
        }
      } else {  // lfL2L
        separable(o, o.l2l, v, Lexp(o, c, 0), res.data());
        cplx* Lc = Lexp(o, t, 0);
        for (int l = 0; l < LL; l++) Lc[l] += res[l];
      }
    }
    downward(o, ti, p);
  }
}

int prcmpt(Oracle& o, bool lists_only = false);
int prcmpt(Oracle& o, bool lists_only) {
  init_circulant(o);
  int st = init_frequency(o);
  if (st) return st;
  init_signatures(o);
  init_interp(o);
  std::vector<std::vector<char>> teff(o.T.cells.size()), seff(o.S.cells.size());
  for (size_t i = 0; i < o.T.cells.size(); i++)
    if (o.prec[o.T.cells[i].lvl] && o.isHF[o.T.cells[i].lvl])
      teff[i].assign(o.nDir[o.T.cells[i].lvl], 0);
  for (size_t i = 0; i < o.S.cells.size(); i++)
    if (o.prec[o.S.cells[i].lvl] && o.isHF[o.S.cells[i].lvl])
      seff[i].assign(o.nDir[o.S.cells[i].lvl], 0);
  blank_hrz(o, 0, 0, teff, seff);
  if (!o.noHF) {
    blank_down(o, o.S, 0, seff);
    blank_down(o, o.T, 0, teff);
  }
  o.nsrc_exp = assign_slots(o, o.S, seff);
  o.ntrg_exp = assign_slots(o, o.T, teff);
  if (lists_only) {  // trees, cones, effective directions and lists only
    hrz_lists(o, 0, 0);
    return 0;
  }
  // LF spectra (precompute.hpp:38-76): every sorted fundamental index with
  // max >= 2 inside the level bound
  for (int l = 2; l < o.nlvl; l++) {
    if (!(o.prec[l] && !o.isHF[l])) continue;
    double locrad = o.box_rad / (double)(1 << l);
    int m = o.nCellMax[l];
    for (int pi = 0; pi < m * m * m; pi++) {
      int iV[3] = {pi / (m * m), (pi / m) % m, pi % m};
      bool b = false;
      for (int k = 0; k < 3; k++) b = b || iV[k] >= 2;
      for (int k = 0; k < 2; k++) b = b && iV[k] >= iV[k + 1];
      if (!b) continue;
      double fV[3];
      for (int k = 0; k < 3; k++) fV[k] = 2. * (double)iV[k] * locrad;
      o.m2l[std::make_pair(l, (long)pi)] = transfer_spectrum(o, locrad, fV);
    }
  }
  init_leaves(o, o.S, true);
  init_leaves(o, o.T, false);
  hrz_lists(o, 0, 0);
  return 0;
}

void gemv(Oracle& o, const cplx* q_user, cplx* p_user) {
  const int LL = o.LL, PP = o.PP;
  std::vector<cplx> q(o.S.parts.size()), p(o.T.parts.size(), 0.);
  for (size_t i = 0; i < q.size(); i++) q[i] = q_user[o.S.parts[i].ind];
  o.Ms.assign((size_t)o.nsrc_exp * LL, 0.);
  o.Fs.assign((size_t)o.nsrc_exp * PP, 0.);
  o.Ls.assign((size_t)o.ntrg_exp * LL, 0.);
  o.Js.assign((size_t)o.ntrg_exp * PP, 0.);
  upward(o, 0, q.data());
  // m2fpass.hpp:38-48 + circulant.hpp:96-106: pad at itilda, forward DFT
  parallel_for(o.nsrc_exp, 64, [&](long e) {
    cplx* F = &o.Fs[e * PP];
    const cplx* M = &o.Ms[e * LL];
    for (int i = 0; i < LL; i++) F[o.itilda[i]] = M[i];
    o.dft.run(F, true);
  });
  // M2L (M2L.hpp:115-157), target-stationary per far pair
  {
    const size_t nh = o.far_hf.size() / 6, nl = o.far_lf.size() / 5;
    std::vector<std::vector<size_t>> by_t(o.T.cells.size());
    for (size_t r = 0; r < nh; r++) by_t[o.far_hf[6 * r]].push_back(r);
    for (size_t r = 0; r < nl; r++) by_t[o.far_lf[5 * r]].push_back(nh + r);
    parallel_for((long)by_t.size(), 16, [&](long ti) {
      for (size_t r : by_t[ti]) {
        const Cell& t = o.T.cells[ti];
        int si, lvl, cone = -1, hsh;
        long iz;
        if (r < nh) {
          const int32_t* f = &o.far_hf[6 * r];
          si = f[1], lvl = f[2], cone = f[3], iz = f[4], hsh = f[5];
        } else {
          const int32_t* f = &o.far_lf[5 * (r - nh)];
          si = f[1], lvl = f[2], iz = f[3], hsh = f[4];
        }
        const Cell& s = o.S.cells[si];
        const cplx* u = o.m2l.at(std::make_pair(lvl, iz)).data();
        const int* pm = o.perm[hsh].data();
        const cplx* y = cone >= 0 ? Fexp(o, s, s.slot[cone] - 1) : Fexp(o, s, 0);
        cplx* x = cone >= 0 ? Jexp(o, t, t.slot[cone] - 1) : Jexp(o, t, 0);
        for (int i = 0; i < PP; i++) x[i] += u[pm[i]] * y[i];
      }
    });
  }
  // P2P (P2P.hpp:43-79 arithmetic), grouped by target cell
  {
    std::vector<std::vector<int>> by_t(o.T.cells.size());
    for (size_t r = 0; r < o.near.size() / 2; r++) by_t[o.near[2 * r]].push_back(o.near[2 * r + 1]);
    // targets of different pairs may overlap (a non-leaf target spans its
    // leaves), so accumulate per pair into a private buffer per thread
    // a non-leaf target spans its leaves, so pairs of different target
    // cells can hit the same particles: accumulate into one buffer per leaf
    // owner -- here simply serialise per target subtree by locking.
    std::vector<cplx> acc(p.size(), 0.);
    std::mutex mu;
    parallel_for((long)by_t.size(), 16, [&](long ti) {
      if (by_t[ti].empty()) return;
      const Cell& t = o.T.cells[ti];
      std::vector<cplx> mine(t.nprt, 0.);
      Cell tl = t;
      tl.first = 0;
      for (int si : by_t[ti]) {
        // p2p accumulates into p[t.first + i]; use a local window
        std::vector<cplx> win(t.nprt, 0.);
        const double pi4m1 = 1. / kPi4;
        const Cell& s = o.S.cells[si];
        for (int i = 0; i < t.nprt; i++) {
          const double* pt = o.T.parts[t.first + i].pos;
          double pr = 0., pim = 0.;
          for (int j = 0; j < s.nprt; j++) {
            const double* ps = o.S.parts[s.first + j].pos;
            double qr = q[s.first + j].real(), qi = q[s.first + j].imag();
            double x = pt[0] - ps[0], y = pt[1] - ps[1], z = pt[2] - ps[2];
            double R = x * x + y * y + z * z;
            double K = 1. / std::sqrt(R);
            if (R < 1.e-16) K = 0.;
            double r = K * R;
            r *= o.kappa;
            K *= pi4m1;
            double co = std::cos(r) * K, si2 = std::sin(r) * K;
            pr += co * qr - si2 * qi;
            pim += co * qi + si2 * qr;
          }
          mine[i] += cplx(pr, pim);
        }
      }
      std::lock_guard<std::mutex> g(mu);
      for (int i = 0; i < t.nprt; i++) acc[t.first + i] += mine[i];
    });
    for (size_t i = 0; i < p.size(); i++) p[i] += acc[i];
  }
  // f2lpass.hpp:36-45 + circulant.hpp:109-118: backward DFT, gather, /PP
  parallel_for(o.ntrg_exp, 64, [&](long e) {
    std::vector<cplx> tmp(o.Js.begin() + e * PP, o.Js.begin() + (e + 1) * PP);
    o.dft.run(tmp.data(), false);
    cplx* Lx = &o.Ls[e * LL];
    for (int i = 0; i < LL; i++) Lx[i] += tmp[o.itilda[i]] / (double)PP;
  });
  downward(o, 0, p.data());
  for (size_t i = 0; i < p.size(); i++) p_user[o.T.parts[i].ind] = p[i];
}

}  // namespace

// =================================================================== C ABI ==
extern "C" {

void* oracle_create_opt(const double* src, int64_t ns, const double* trg, int64_t nt,
                        int L, int ncrit, double kappa, int lvmax, int lists_only);
void* oracle_create(const double* src, int64_t ns, const double* trg, int64_t nt,
                    int L, int ncrit, double kappa, int lvmax) {
  return oracle_create_opt(src, ns, trg, nt, L, ncrit, kappa, lvmax, 0);
}

// lists_only != 0: prcmpt stops after the trees, cones, effective directions
// and interaction lists (no leaf matrices, no LF spectra): enough to pin
// those at sizes whose full precomputation does not fit in host memory.
void* oracle_create_opt(const double* src, int64_t ns, const double* trg, int64_t nt,
                        int L, int ncrit, double kappa, int lvmax, int lists_only) {
  Oracle* o = new Oracle;
  o->L = L;
  o->P = 2 * L - 1;
  o->LL = L * L * L;
  o->PP = o->P * o->P * o->P;
  o->ncrit = ncrit;
  o->lvmax = lvmax;
  o->kappa = kappa;
  if (ns <= 0 || nt <= 0 || L < 2 || L > 8) {
    o->status = -1;
    return o;
  }
  o->S.parts.resize(ns);
  o->T.parts.resize(nt);
  for (int64_t i = 0; i < ns; i++) {
    for (int k = 0; k < 3; k++) o->S.parts[i].pos[k] = src[3 * i + k];
    o->S.parts[i].ind = (int)i;
  }
  for (int64_t i = 0; i < nt; i++) {
    for (int k = 0; k < 3; k++) o->T.parts[i].pos[k] = trg[3 * i + k];
    o->T.parts[i].ind = (int)i;
  }
  get_bounds(o->T.parts, o->S.parts, o->box_ctr, o->box_rad);
  int id0[3] = {0, 0, 0};
  for (Tree* t : {&o->T, &o->S}) {
    Builder b{&t->parts, &t->cells, ncrit, lvmax};
    b.build(0, (int)t->parts.size(), o->box_ctr, o->box_rad, id0, 0);
    if (b.overflow) {
      o->status = -2;
      return o;
    }
  }
  o->status = prcmpt(*o, lists_only != 0);
  return o;
}

// Order-independent digest of n records of w int32 fields: out = {n,
// sum of h1(record), sum of h2(record)} mod 2^64, h1 / h2 two seeded
// splitmix64 chains over the fields.  Equal multisets of records give equal
// digests; a changed, missing or extra record changes both sums.
static uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
void oracle_digest_records(const int32_t* rec, int64_t n, int w, uint64_t* out) {
  std::atomic<uint64_t> a1(0), a2(0);
  const long nb = (long)((n + 65535) / 65536);
  parallel_for(nb, 1, [&](long b) {
    uint64_t s1 = 0, s2 = 0;
    const int64_t e = std::min<int64_t>(n, (int64_t)(b + 1) * 65536);
    for (int64_t i = (int64_t)b * 65536; i < e; i++) {
      uint64_t h1 = 0x243f6a8885a308d3ULL, h2 = 0x13198a2e03707344ULL;
      for (int k = 0; k < w; k++) {
        const uint64_t v = (uint64_t)(uint32_t)rec[i * w + k];
        h1 = mix64(h1 ^ v);
        h2 = mix64(h2 + v * 0xa4093822299f31d0ULL);
      }
      s1 += h1;
      s2 += h2;
    }
    a1 += s1;
    a2 += s2;
  });
  out[0] = (uint64_t)n;
  out[1] = a1.load();
  out[2] = a2.load();
}

// The same digest of the oracle's own lists: which 0 near (2 fields),
// 1 far HF (6 fields), 2 far LF (5 fields).
void oracle_lists_digest(void* h, int which, uint64_t* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const std::vector<int32_t>& v = which == 0 ? o->near : which == 1 ? o->far_hf : o->far_lf;
  const int w = which == 0 ? 2 : which == 1 ? 6 : 5;
  oracle_digest_records(v.data(), (int64_t)v.size() / w, w, out);
}

int oracle_status(void* h) { return static_cast<Oracle*>(h)->status; }
void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }

int oracle_gemv(void* h, const double* q, double* p) {
  Oracle* o = static_cast<Oracle*>(h);
  if (o->status) return o->status;
  gemv(*o, reinterpret_cast<const cplx*>(q), reinterpret_cast<cplx*>(p));
  return 0;
}

// info: 0 nlvl, 1 cpt, 2 max_stage, 3 n far_hf, 4 n far_lf, 5 n near,
// 6 cells T, 7 cells S, 8 nsrc_exp, 9 ntrg_exp, 10 n HF tables
int64_t oracle_info(void* h, int what) {
  Oracle* o = static_cast<Oracle*>(h);
  switch (what) {
    case 0: return o->nlvl;
    case 1: return o->cpt;
    case 2: return o->max_stage;
    case 3: return (int64_t)o->far_hf.size() / 6;
    case 4: return (int64_t)o->far_lf.size() / 5;
    case 5: return (int64_t)o->near.size() / 2;
    case 6: return (int64_t)o->T.cells.size();
    case 7: return (int64_t)o->S.cells.size();
    case 8: return o->nsrc_exp;
    case 9: return o->ntrg_exp;
    case 10: {
      int64_t n = 0;
      for (auto& kv : o->m2l) n += o->isHF[kv.first.first] ? 1 : 0;
      return n;
    }
  }
  return -1;
}

// Same record layouts as oracle/ref_harness.cpp.
void oracle_cells(void* h, int which, int32_t* ci, double* cd) {
  Oracle* o = static_cast<Oracle*>(h);
  const Tree& t = which ? o->S : o->T;
  for (size_t i = 0; i < t.cells.size(); i++) {
    const Cell& c = t.cells[i];
    int32_t r[8] = {c.idx[0], c.idx[1], c.idx[2], c.lvl, c.nprt, c.first,
                    (int32_t)c.son.size(), c.nexp};
    std::memcpy(ci + 8 * i, r, sizeof r);
    cd[4 * i] = c.ctr[0];
    cd[4 * i + 1] = c.ctr[1];
    cd[4 * i + 2] = c.ctr[2];
    cd[4 * i + 3] = c.rad;
  }
}
int64_t oracle_dirs(void* h, int which, int32_t* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const Tree& t = which ? o->S : o->T;
  int64_t n = 0;
  for (auto& c : t.cells)
    for (int d : c.dirs) {
      if (out) out[n] = d;
      n++;
    }
  return n;
}
void oracle_perm(void* h, int which, int32_t* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const Tree& t = which ? o->S : o->T;
  for (size_t i = 0; i < t.parts.size(); i++) out[i] = t.parts[i].ind;
}
void oracle_lists(void* h, int32_t* near, int32_t* far_hf, int32_t* far_lf) {
  Oracle* o = static_cast<Oracle*>(h);
  std::memcpy(near, o->near.data(), o->near.size() * 4);
  std::memcpy(far_hf, o->far_hf.data(), o->far_hf.size() * 4);
  std::memcpy(far_lf, o->far_lf.data(), o->far_lf.size() * 4);
}
// HF transfer spectrum of (lvl, iz) as built by blankM2Lhf; returns 0 if absent
int oracle_table(void* h, int lvl, int64_t iz, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  auto it = o->m2l.find(std::make_pair(lvl, (long)iz));
  if (it == o->m2l.end()) return 0;
  std::memcpy(out, it->second.data(), it->second.size() * 16);
  return 1;
}
void oracle_direction(void* h, int stage, int d, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  for (int k = 0; k < 3; k++) out[k] = o->D.tab[stage][d][k];
}

// FP64 direct sum (interface.hpp:178-221 arithmetic) at selected targets.
void oracle_direct(const double* src, int64_t ns, const double* q,
                   const double* trg, int64_t nt, double kappa, double* out) {
  const double pi4m1 = 1. / kPi4;
  parallel_for(nt, 8, [&](long i) {
    double pr = 0., pim = 0.;
    for (int64_t j = 0; j < ns; j++) {
      double x = trg[3 * i] - src[3 * j], y = trg[3 * i + 1] - src[3 * j + 1],
             z = trg[3 * i + 2] - src[3 * j + 2];
      double R = x * x + y * y + z * z;
      double K = 1. / std::sqrt(R);
      if (R < 1.e-16) K = 0.;
      double r = K * R * kappa;
      K *= pi4m1;
      double co = std::cos(r) * K, si = std::sin(r) * K;
      pr += co * q[2 * j] - si * q[2 * j + 1];
      pim += co * q[2 * j + 1] + si * q[2 * j];
    }
    out[2 * i] = pr;
    out[2 * i + 1] = pim;
  });
}

}  // extern "C"
