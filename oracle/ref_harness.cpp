// Test infrastructure (oracle only, never shipped): a driver that compiles the
// reference defmm headers UNMODIFIED (include path points at the read-only
// reference checkout) and runs its own public API, exactly like the
// reference's test/testinterface.cpp:13-34:
//
//   IBFMM_Mat<3> A;  A.addSourceParticle(..);  A.addTargetParticle(..);
//   A.prcmpt(L, Ncrit, kappa, lvMAX);  gemv(A, In, Out);
//
// It then dumps what the reference built (both trees, effective directions,
// far/near interaction lists with their cones) and the potentials, so that
// the restated oracle and the CUDA path can be pinned against the reference.
//
// The far/near lists are re-enumerated with the reference's own predicates
// (MACgeomhf, MAClist, isLeaf, chooseM2Lhf/chooseM2L; hrzpass.hpp:40-91,
// M2L.hpp:88-112) in the same DFS order as HorizontalPass (hrzpass.hpp:62-91).
//
// Input  (argv[1]): binary file, see write_case() in oracle/refrun.py.
// Output (argv[2]): directory receiving raw little-endian arrays + summary.txt.
#include "interface.hpp"

#include <chrono>
#include <cstdio>
#include <cstdint>
#include <string>
#include <vector>

using namespace defmm;

namespace {

struct Header {
  char magic[8];
  int64_t nS, nT;
  int32_t L, Ncrit, lvMAX, flags;
  double kappa;
};

std::vector<int32_t> g_near, g_far_hf, g_far_lf;

void enumerate(int i, int j, cell<3>* X, cell<3>* Y) {
  if (global::precomputationAtStage[X[i].lvl] && X[i].lvl == Y[j].lvl) {
    if ((X + i)->lvl && global::isHFStage[(X + i)->lvl]) {
      if (MACgeomhf(X[i], Y[j])) {
        veci<3> iZ = X[i].idx - Y[j].idx;
        int iobc = -1;
        cplx* u = nullptr;
        int* perm = chooseM2Lhf(X[i].lvl, iZ, &u, &iobc);
        (void)perm;
        veci<3> nI;
        int hsh;
        int* p2;
        getPermuteAndFundamentalMultiIndexAndHashcode(iZ, nI, p2, hsh);
        int iz = thetis::keys::I2i<3>(nI, global::nCellPerDirMax[X[i].lvl]);
        int32_t rec[6] = {i, j, X[i].lvl, iobc, iz, hsh};
        g_far_hf.insert(g_far_hf.end(), rec, rec + 6);
        return;
      }
    } else {
      if (MAClist(X[i], Y[j])) {
        veci<3> iZ = X[i].idx - Y[j].idx;
        veci<3> nI;
        int hsh;
        int* p2;
        getPermuteAndFundamentalMultiIndexAndHashcode(iZ, nI, p2, hsh);
        int iz = thetis::keys::I2i<3>(nI, global::nCellPerDirMax[X[i].lvl]);
        int32_t rec[5] = {i, j, X[i].lvl, iz, hsh};
        g_far_lf.insert(g_far_lf.end(), rec, rec + 5);
        return;
      }
    }
  }
  if (isLeaf(X[i]) || isLeaf(Y[j])) {
    g_near.push_back(i);
    g_near.push_back(j);
    return;
  }
  for (unsigned k1 = 0; k1 < X[i].son.size(); k1++)
    for (unsigned k2 = 0; k2 < Y[j].son.size(); k2++)
      enumerate(X[i].son[k1], Y[j].son[k2], X, Y);
}

template <typename T>
void dump(const std::string& path, const std::vector<T>& v) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::perror(path.c_str());
    std::exit(2);
  }
  if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
  std::fclose(f);
}

int count_cells(cell<3>* root) {
  // DFS pre-order array: every cell is reachable from cell 0 through `son`.
  int n = 0;
  std::vector<int> stack{0};
  while (!stack.empty()) {
    int c = stack.back();
    stack.pop_back();
    n++;
    for (int s : root[c].son) stack.push_back(s);
  }
  return n;
}

void dump_tree(const std::string& dir, const char* tag, cell<3>* root) {
  const int n = count_cells(root);
  std::vector<int32_t> ci, sons, dirs, perm;
  std::vector<double> cd;
  for (int c = 0; c < n; c++) {
    const cell<3>& x = root[c];
    const bool prec = global::precomputationAtStage[x.lvl];
    const bool hf = prec && global::isHFStage[x.lvl];
    const int nexp = hf ? x.ndir : (prec ? 1 : 0);
    int32_t rec[8] = {x.idx[0], x.idx[1], x.idx[2], x.lvl,
                      x.nprt,   x.ind,    (int32_t)x.son.size(), nexp};
    ci.insert(ci.end(), rec, rec + 8);
    cd.push_back(x.ctr[0]);
    cd.push_back(x.ctr[1]);
    cd.push_back(x.ctr[2]);
    cd.push_back(x.rad);
    for (int s : x.son) sons.push_back(s);
    if (hf)
      for (int k = 0; k < x.ndir; k++) dirs.push_back(x.dirs[k]);
  }
  for (int i = 0; i < root[0].nprt; i++) perm.push_back(root[0].prt[i].ind);
  dump(dir + "/cells_" + tag + "_int.bin", ci);
  dump(dir + "/cells_" + tag + "_dbl.bin", cd);
  dump(dir + "/sons_" + tag + ".bin", sons);
  dump(dir + "/dirs_" + tag + ".bin", dirs);
  dump(dir + "/perm_" + tag + ".bin", perm);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s case.bin outdir [nolists]\n", argv[0]);
    return 2;
  }
  const bool lists = !(argc > 3 && std::string(argv[3]) == "nolists");
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) {
    std::perror(argv[1]);
    return 2;
  }
  Header h;
  if (std::fread(&h, sizeof(h), 1, f) != 1 ||
      std::string(h.magic, 8) != "DFMMIN01") {
    std::fprintf(stderr, "bad case file\n");
    return 2;
  }
  std::vector<double> ys(3 * h.nS), xs(3 * h.nT), q(2 * h.nS);
  if (std::fread(ys.data(), 8, ys.size(), f) != ys.size() ||
      std::fread(xs.data(), 8, xs.size(), f) != xs.size() ||
      std::fread(q.data(), 8, q.size(), f) != q.size()) {
    std::fprintf(stderr, "short case file\n");
    return 2;
  }
  std::fclose(f);
  const std::string out = argv[2];

  IBFMM_Mat<3> A;
  for (int64_t i = 0; i < h.nS; i++) A.addSourceParticle(&ys[3 * i]);
  for (int64_t i = 0; i < h.nT; i++) A.addTargetParticle(&xs[3 * i]);
  Vecc In(h.nS), Out(h.nT);
  Out = cplx0;
  for (int64_t i = 0; i < h.nS; i++) In[i] = cplx(q[2 * i], q[2 * i + 1]);

  auto t0 = std::chrono::steady_clock::now();
  A.prcmpt(h.L, h.Ncrit, h.kappa, h.lvMAX);
  auto t1 = std::chrono::steady_clock::now();
  gemv(A, In, Out);
  auto t2 = std::chrono::steady_clock::now();

  std::vector<double> pot(2 * h.nT);
  for (int64_t i = 0; i < h.nT; i++) {
    pot[2 * i] = Out[i].real();
    pot[2 * i + 1] = Out[i].imag();
  }
  dump(out + "/pot.bin", pot);
  dump_tree(out, "S", SourceRoot(A));
  dump_tree(out, "T", TargetRoot(A));
  if (lists) {
    enumerate(0, 0, TargetRoot(A), SourceRoot(A));
    dump(out + "/near.bin", g_near);
    dump(out + "/far_hf.bin", g_far_hf);
    dump(out + "/far_lf.bin", g_far_lf);
  }
  FILE* s = std::fopen((out + "/summary.txt").c_str(), "w");
  std::fprintf(s, "prcmpt_s=%.9f\n",
               std::chrono::duration<double>(t1 - t0).count());
  std::fprintf(s, "gemv_s=%.9f\n",
               std::chrono::duration<double>(t2 - t1).count());
  std::fprintf(s, "hf_tables=%d\n", hrzpassinternal::cpt);
  std::fprintf(s, "kappa=%.17g\n", global::kappa);
  std::fclose(s);
  return 0;
}
