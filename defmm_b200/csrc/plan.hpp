// Host-side plan of one directional FMM operator: octrees, frequency regime,
// direction (cone) tables, interaction lists, expansion slots and transfer
// spectra, laid out for the device kernels.
//
// Everything here follows the semantics of IChollet/defmm's precomputation
// (include/interface.hpp:100-151) bit-exactly where the result is discrete
// (trees, admissibility, cones, effective directions); the construction itself
// is level-wise and multi-threaded instead of the reference's recursions.
#pragma once

#include <array>
#include <chrono>
#include <complex>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace dfb {

// exp(-2 pi i m / P), m < P, as (re, im) pairs: the twiddles of the plan's
// forward DFTs (computed in long double, rounded once).
void dft_twiddles(int P, double* w);
// Node i of the equispaced grid of order L on [-alpha, alpha].
double node_coord(int i, int L, double alpha);

// Seconds on a monotonic clock (setup step timing).
inline double wall_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

typedef std::complex<double> cplx;

// One octree, cells in depth-first pre-order (the reference's cell array
// order, sort.hpp:187-220), particles in tree order.
struct Tree {
  int64_t ncell = 0;
  int nlvl = 0;
  std::vector<int32_t> idx;        // 3 per cell: integer coordinates at its level
  std::vector<int32_t> lvl, nprt, first, parent, nson;
  std::vector<int64_t> son_ptr;    // CSR into sons (ncell + 1)
  std::vector<int32_t> sons;
  std::vector<int32_t> sub_end;    // one past the last cell of the subtree (DFS)
  std::vector<double> ctr;         // 3 per cell
  std::vector<double> rad;
  std::vector<int32_t> perm;       // tree order position -> user index
  std::vector<double> pos;         // 3 per particle, tree order
  std::vector<int64_t> lvl_cells;  // cells per level
  bool leaf(int64_t c) const { return nson[c] == 0; }
};

// Per-level frequency regime (frequency.hpp:44-184).
struct Levels {
  int nlvl = 0, cpt = 0, max_stage = 0;
  bool noHF = true;
  std::vector<int> isHF, HFStage, nDir, nCellMax;
  std::vector<char> prec;
};

// Expansion slots of one tree: one per (cell, effective direction) at
// precomputed HF levels, one per cell at precomputed LF levels.  Slots are
// ordered level-major, then cone-major, then by cell (DFS order), so one cone
// of one level is a contiguous slot range.
struct Slots {
  int64_t n = 0;
  std::vector<int32_t> cell, dir;          // per slot (dir = -1 for LF)
  std::vector<int64_t> lvl_begin;          // nlvl + 1
  std::vector<std::vector<int64_t>> cone_begin;  // per level: nDir + 1 offsets
  // per cell: effective directions in increasing order with their slots
  std::vector<int64_t> cell_ptr;           // ncell + 1 into cell_dirs / cell_slots
  std::vector<int32_t> cell_dirs;
  std::vector<int64_t> cell_slots;
  int64_t slot_of(int64_t c, int d) const;  // -1 when absent; d = -1 for LF
};

struct Plan {
  // parameters
  int L = 0, P = 0, LL = 0, PP = 0, ncrit = 0, lvmax = -1;
  double kappa = 0.;
  double box_ctr[3] = {0, 0, 0}, box_rad = 0.;
  Tree S, T;
  Levels lv;
  // direction tables per HF stage: 6*4^e unit vectors (newdirections.hpp:76-171)
  std::vector<std::vector<double>> dirs;  // [stage][3*i]
  // plane-wave signature grids per HF stage (planewave.hpp:44-69): [stage][d*LL + k]
  std::vector<std::vector<cplx>> sig, sig2;
  // separable interpolation matrices (interpolation.hpp:184-242), L x L column-major
  std::vector<double> m2m[2], l2l[2];
  // circulant embedding (circulant.hpp:47-93) and spectrum permutations
  // (permutations.hpp:128-150)
  std::vector<int32_t> itilda;             // LL
  std::vector<double> tabZ;                // 3*PP
  std::vector<uint16_t> perm;              // 64*PP
  Slots sS, sT;
  // transfer spectra: one per distinct (level, fundamental index)
  std::vector<int32_t> tab_lvl;
  std::vector<int64_t> tab_iz;
  std::vector<cplx> tables;                // ntab * PP
  // M2L, grouped by target slot (CSR over target slots)
  std::vector<int64_t> m2l_ptr;            // sT.n + 1
  std::vector<int32_t> m2l_src;            // source slot
  std::vector<uint32_t> m2l_tab;           // permuted spectrum id (index into ptab_key)
  // permuted spectra actually used: (table index << 6) | hash; the device
  // holds U_k[i] = tables[key >> 6][perm[key & 63][i]]
  std::vector<uint32_t> ptab_key;
  // M2L entries already on the device (built there by the level walk):
  // int32 source slots and uint32 permuted-spectrum ids, n_m2l each, in
  // m2l_ptr order; the host copies m2l_src / m2l_tab stay empty.  The
  // operator that owns the plan releases them.
  void* dev_m2l_src = nullptr;
  void* dev_m2l_tab = nullptr;
  int64_t n_m2l = 0;
  // M2M / L2L transfer lists built by the device walk and left there: int64
  // pointers over the source / target slots (n + 1) and int32 entries
  // (n_m2m / n_l2l); m2m_ptr, m2m_child, l2l_ptr, l2l_parent stay empty.
  void *dev_m2m_ptr = nullptr, *dev_m2m_child = nullptr, *dev_l2l_ptr = nullptr, *dev_l2l_parent = nullptr;
  int64_t n_m2m = 0, n_l2l = 0;
  // Per-cell slot lists built by the device walk: int32 slot ids and
  // directions in Slots::cell_ptr order, left on the device (sT / sS keep
  // cell_ptr and cell_dirs on the host, cell_slots stays empty); with them
  // the slots' own cells and directions (Slots::cell, dir), also on the host
  void *dev_cslot_T = nullptr, *dev_cdir_T = nullptr, *dev_cslot_S = nullptr, *dev_cdir_S = nullptr;
  void *dev_scell_T = nullptr, *dev_sdir_T = nullptr, *dev_scell_S = nullptr, *dev_sdir_S = nullptr;
  // M2M children of each source slot, L2L parents of each target slot
  std::vector<int64_t> m2m_ptr;            // sS.n + 1
  std::vector<int32_t> m2m_child;          // child slot
  std::vector<int64_t> l2l_ptr;            // sT.n + 1
  std::vector<int32_t> l2l_parent;         // parent slot
  // leaves at precomputed levels (P2M sources / L2P targets)
  std::vector<int32_t> p2m_leaf, l2p_leaf;
  // near field, grouped by target leaf chunk (<= 32 targets per chunk); a
  // chunk's source ranges are cut into work items of at most kItemSources
  // sources (a coarse leaf next to a large subtree can meet most of the
  // points), each item yields partial sums for its chunk's targets, added per
  // chunk in item order
  static constexpr int kItemSources = 8192;
  std::vector<int32_t> p2p_tfirst, p2p_tn;   // per chunk
  std::vector<int64_t> p2p_ptr;              // items + 1
  std::vector<int32_t> p2p_sfirst, p2p_sn;   // source particle ranges
  std::vector<int32_t> p2p_item_chunk;       // per item
  std::vector<int64_t> p2p_chunk_items;      // chunks + 1 (a chunk's items are consecutive)
  std::vector<int32_t> p2p_order;            // items by decreasing work
  // Symmetric near field (sources and targets are the same points, so the
  // particle interactions come in mirrored pairs): each chunk keeps its own
  // leaf as a plain block (self_*) and the source leaves after its leaf in
  // tree order as symmetric blocks (sym_*); one evaluation of G(x_i, y_j)
  // then serves p_i and p_j.  The mirrored part (sources before the leaf)
  // is dropped: it arrives from the other leaf's chunks, as partial sums
  // written to scratch at sym_soff and reduced per source leaf (red_*) in a
  // fixed order.
  bool p2p_sym = false;
  std::vector<int64_t> self_ptr;             // chunks + 1
  std::vector<int32_t> self_sfirst, self_sn, self_order;
  std::vector<int64_t> sym_ptr;              // items + 1 into sym ranges
  std::vector<int32_t> sym_sfirst, sym_sn, sym_order;
  std::vector<int64_t> sym_soff;             // scratch slot of the range's first source
  std::vector<int32_t> sym_item_chunk;       // per item
  std::vector<int64_t> sym_chunk_items;      // chunks + 1
  // per source leaf receiving partial sums: its particles and the scratch
  // rows to add (row k covers the leaf's particles at red_off[k] + j)
  std::vector<int32_t> red_first, red_n;
  std::vector<int64_t> red_ptr, red_off;     // leaves + 1 into red_off (chunk order)
  int64_t sym_scratch = 0;                   // scratch slots (one complex each)
  // The same near-field lists built on the device by the device walk (the
  // host vectors p2p_*, self_*, sym_*, red_* above then stay empty): device
  // arrays with the host build's contents, and their sizes.  The operator
  // that owns the plan releases them (dev_near_allocs).
  struct NearOnDevice {
    bool on = false;
    int64_t nchunk = 0, p2p_items = 0, n_self_order = 0, sym_items = 0, n_red = 0;
    const int32_t *tfirst = nullptr, *tn = nullptr;
    const int64_t *p2p_ptr = nullptr, *p2p_chunk_items = nullptr;
    const int32_t *p2p_sfirst = nullptr, *p2p_sn = nullptr, *p2p_item_chunk = nullptr, *p2p_order = nullptr;
    const int64_t *self_ptr = nullptr;
    const int32_t *self_sfirst = nullptr, *self_sn = nullptr, *self_order = nullptr;
    const int64_t *sym_ptr = nullptr, *sym_soff = nullptr, *sym_chunk_items = nullptr;
    const int32_t *sym_sfirst = nullptr, *sym_sn = nullptr, *sym_item_chunk = nullptr, *sym_order = nullptr;
    const int32_t *red_first = nullptr, *red_n = nullptr;
    const int64_t *red_ptr = nullptr, *red_off = nullptr;
  } nd;
  std::vector<void*> dev_near_allocs;
  // sizes of the near-field lists wherever they were built
  int64_t near_chunks() const { return nd.on ? nd.nchunk : (int64_t)p2p_tfirst.size(); }
  int64_t near_items() const { return nd.on ? nd.p2p_items : (int64_t)p2p_order.size(); }
  int64_t near_self_items() const { return nd.on ? nd.n_self_order : (int64_t)self_order.size(); }
  int64_t near_sym_items() const { return nd.on ? nd.sym_items : (int64_t)sym_order.size(); }
  int64_t near_red_leaves() const { return nd.on ? nd.n_red : (int64_t)red_first.size(); }
  // statistics
  int64_t n_far_hf = 0, n_far_lf = 0, n_near = 0, i_near = 0;
  // Optional record of the lists for parity checks: far (t, s, lvl, cone,
  // iz, hash) and near (t, s) in the reference's HorizontalPass order.
  bool keep_lists = false;
  std::vector<int32_t> rec_far_hf, rec_far_lf, rec_near;
  double t_tree = 0, t_lists = 0, t_tables = 0, t_walk = 0;  // t_walk: part of t_lists
  // wall time of each setup step, in order (name, seconds)
  std::vector<std::pair<const char*, double>> t_steps;
  void step(const char* name, double& t0) {  // records now - t0 and resets t0
    const double t = wall_seconds();
    t_steps.push_back({name, t - t0});
    t0 = t;
  }
  bool tree_on_device = false;  // the octrees' particle ordering ran on the device
  // Transfer spectra and signatures left to the device (device_plan_tables):
  // `tables` and the values of sig/sig2 stay empty (sig/sig2 keep their
  // sizes), tab_fund holds each table's fundamental index.
  bool tables_on_device = false;
  std::vector<std::array<int32_t, 3>> tab_fund;
};

// Result of the level-by-level dual traversal (hrzpass.hpp:62-143 with the
// blank passes, dwnpass.hpp:81-109): besides what it fills in the plan (slots
// sS/sT without their per-cell CSR, tab_lvl/tab_iz, far counts, list
// records), the far entries of every level and the near pairs, both in the
// reference's depth-first order.
struct LevelWalk {
  std::vector<std::pair<int32_t, int32_t>> near_pairs;
  std::vector<std::array<int32_t, 3>> tab_nI;  // fundamental index per table
  std::vector<std::vector<int32_t>> far_ts, far_ss;  // per level: slots
  std::vector<std::vector<uint32_t>> far_tab;        // per level: (table << 6) | hash
  // Set by a walker that also grouped the far entries by target slot itself
  // (the M2L CSR with permuted-spectrum ids): it fills Plan::m2l_ptr and
  // ptab_key and leaves the entries in Plan::dev_m2l_src / dev_m2l_tab.
  bool m2l_done = false;
  // Set by a walker that also built the M2M / L2L transfer lists (on the
  // device: Plan::dev_m2m_ptr etc.).
  bool transfers_done = false;
  // Set by a walker that also built the per-cell slot lists (cell_ptr and
  // cell_dirs on the host, slot ids on the device: Plan::dev_cslot_T etc.).
  bool cells_done = false;
  // Set by a walker that also built the near-field lists (on the device:
  // Plan::nd, with Plan::n_near and i_near); near_pairs then stays empty.
  bool near_done = false;
};

// Another implementation of the level walk (the device one); it must produce
// exactly the host walk's results.  Returns 0 or a negative status.
struct LevelWalker {
  virtual ~LevelWalker() = default;
  virtual int walk(Plan& p, LevelWalk& w, std::string& err) = 0;
};

// The particle ordering of the octree build on another processor (the
// device one, plan_device.cu).  The host keeps the cells and decides which
// split; per level the sorter returns the octant counts of the splitting
// cells' particles (bit code sum_k (x_k > c_k) << k, the cell centres given
// by the host) and then moves every particle of a splitting cell to its
// child's range, stably; at the end it returns the final order.  The cells
// and the order are then exactly the host build's.
struct TreeSorter {
  virtual ~TreeSorter() = default;
  virtual int begin(const double* pts, int64_t n, std::string& err) = 0;
  // m cells of the level: first particle position, centre (3 per cell),
  // split flag; hist: m x 8 octant counts (zero for cells that stay)
  virtual int histogram(int64_t m, const int64_t* first, const double* ctr, const uint8_t* split, int64_t* hist,
                        std::string& err) = 0;
  // first position of each (cell, octant) child, -1 where there is none
  virtual int reorder(const int64_t* child_first, std::string& err) = 0;
  virtual int finish(int32_t* order, std::string& err) = 0;
};

// Build the plan; returns 0 or a negative status with `err` set.  With a
// walker (and no list records requested) the level walk runs there; with a
// sorter the octrees' particle ordering runs there.
//   -2: coincident points keep a cell above ncrit (the reference recurses
//       without end, sort.hpp:98-162)
//   -3: the tree is too shallow for any M2L level (frequency.hpp:114-120)
//   -1: invalid arguments
int build_plan(Plan& p, const double* src, int64_t ns, const double* trg,
               int64_t nt, int L, int ncrit, double kappa, int lvmax,
               std::string& err, LevelWalker* walker = nullptr, TreeSorter* sorter = nullptr);

}  // namespace dfb
