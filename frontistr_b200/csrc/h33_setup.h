// h33_setup.h -- host-side symbolic setup of the B200 3x3 solver: orderings, reordered
// profiles, block ILU(0) factorisation and the sliced block-ELL layouts.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace h33 {

// Checks an hecmwST profile of one domain (NP >= N rows, indexX[0..NP] consistent
// with NPL/NPU, itemL ascending ids below the row, itemU ascending ids above it up to
// NP, 1-based).
// Returns "" or the first problem found.
std::string check_profile(int N, int NP, int NPL, int NPU, const int *indexL, const int *itemL,
                          const int *indexU, const int *itemU);

// Borrowed hecmwST_matrix profile (indexX[0..N], itemX 1-based ids).
struct Profile {
  int N;
  const int *indexL, *itemL, *indexU, *itemU;
  int NPL() const { return indexL[N]; }
  int NPU() const { return indexU[N]; }
};

// Raw block numbering used on the device: blocks of D are 0..N-1, AL blocks
// N..N+NPL-1 and AU blocks N+NPL..N+NPL+NPU-1 (the order of the upload buffer).

// Reverse Cuthill-McKee (hecmw_matrix_ordering_CM.f90:18-245).
// perm[new] = old, iperm[old] = new (0-based here).
void ordering_rcm(const Profile &p, std::vector<int> &perm, std::vector<int> &iperm);

// Greedy multicolouring in the order perm_cur (hecmw_matrix_ordering_MC.f90:15-72).
// colorindex has ncolor+1 entries; returns ncolor.
int ordering_mc(const Profile &p, const std::vector<int> &perm_cur, int ncolor_in,
                std::vector<int> &colorindex, std::vector<int> &perm, std::vector<int> &iperm);

// First-fit colouring (each node takes the smallest colour none of its already
// coloured neighbours has) in the input order and in smallest-last order (Matula and
// Beck), whichever needs fewer colours (ties: the input order); rows then ordered by
// colour, by node number inside a colour.  On a structured 27-point mesh numbered
// lexicographically the input order gives the 8 parity colours; on other numberings
// smallest-last usually needs fewer.  Returns the number of colours.
int ordering_greedy(const Profile &p, std::vector<int> &colorindex, std::vector<int> &perm,
                    std::vector<int> &iperm);

// A row-wise list of blocks: for row r, entries [ptr[r], ptr[r+1]) of (col, src),
// col = 0-based node index gathered by the kernel, src = raw block id.
struct BlockRows {
  std::vector<int64_t> ptr;
  std::vector<int> col, src;
};

// Rows of the unified matrix (L, D, U per row, ascending column; raw ids).
void unified_rows(const Profile &p, BlockRows &out);

// SSOR reordering (hecmw_matrix_reorder.f90:20-158): rows in the new order, the
// lower (new col < new row) and upper parts sorted by new column, columns
// renumbered to old node ids, src = raw block id of the value.
void reordered_rows(const Profile &p, const std::vector<int> &perm, const std::vector<int> &iperm,
                    BlockRows &lower, BlockRows &upper);

// Host-side sliced block-ELL layout; rows are taken in groups (a group never
// shares a slice with another group).  Each row is spread over `lanes` lanes of
// a warp (lanes divides 32), so a slice holds 32/lanes consecutive rows: block k
// of the row at offset r sits in slot k/lanes at lane r*lanes + k%lanes, and every
// load of one entry of a slot is 32 consecutive values.
struct SellLayout {
  int nslices = 0;
  int lanes = 1;
  int64_t nslots = 0;
  std::vector<int> row0, nrows, slot0, len;  // per slice
  std::vector<int> rowlen;                    // per slice*32 + row offset (blocks in the row)
  std::vector<int> col, src;                  // per slot*32 + lane (pad: col 0, src -1)
  std::vector<int> group_slice;               // group g -> slices [group_slice[g], group_slice[g+1])
  // run tables (built when max_runs > 0): the slices of group g form runs
  // run_ptr[g] .. run_ptr[g+1]-1 of consecutive slices with one slot count; run i
  // starts at slice group_slice[g] + run_slice[i] and slot run_slot[i] and gives
  // each of its slices run_len[i] slots
  std::vector<int> run_ptr, run_slice, run_slot, run_len;
};
// group_rows: row boundaries of the groups (size ngroups+1, rows 0..nrows-1).
// Each slice gets the largest slot count of its rows.  max_runs > 0: per group, the
// slices' slot counts are raised where needed (padding: column 0, value 0) so that
// they form at most max_runs runs, and the run tables are filled: a kernel then
// finds a slice's first slot and slot count from its index and the group's table.
void build_sell(const BlockRows &rows, const std::vector<int> &group_rows, SellLayout &out,
                int lanes = 1, int max_runs = 0);
// The same layout from the rows' block counts alone (count[r] blocks in row r): every
// field but col and src, which the device fills (block k of the row at offset r of
// slice s goes to slot slot0[s] + k / lanes, lane r * lanes + k % lanes; padding col
// 0, src -1).
void sell_shape(const int *count, const std::vector<int> &group_rows, SellLayout &out, int lanes = 1,
                int max_runs = 0);

// Order of the rows inside each group for the sliced layouts of a lower and an upper
// part with the same rows: sorted by (lower slot count, upper slot count) at `lanes`
// lanes per row, ties in the incoming order, so that the slices of a group need few
// distinct slot counts.  order[new] = old row; rows never leave their group.
void order_rows_by_length(const BlockRows &lower, const BlockRows &upper, const std::vector<int> &group_rows,
                          int lanes, std::vector<int> &order);
// The same from the rows' lower and upper block counts (n rows).
void order_rows_by_counts(const int *nl, const int *nu, int n, const std::vector<int> &group_rows, int lanes,
                          std::vector<int> &order);

// Rows of `in` taken in the order `order` (order[new] = old row) and columns renamed
// by iorder (iorder[old] = new); the blocks of each row keep their order.
void permute_rows(const BlockRows &in, const std::vector<int> &order, const std::vector<int> &iorder,
                  BlockRows &out);

// Element mesh profile (hecmw_mat_con, hecmw1/src/solver/matrix/hecmw_mat_con.f90:21-107):
// per node the sorted, unique lists of lower and upper neighbours over all elements
// sharing it.  conn: n_elem x nn node ids, 1-based.  Outputs 1-based items.
void element_profile(int n_node, int n_elem, int nn, const int *conn, std::vector<int> &indexL,
                     std::vector<int> &itemL, std::vector<int> &indexU, std::vector<int> &itemU);

// For every raw block (D blocks 0..N-1, then AL, then AU) the element contributions
// in element order, as CSR: ptr (nblocks+1) and code = e*nn*nn + a*nn + b (block (a, b)
// of element e).  Throws when the code does not fit in 31 bits.
void element_contributions(int n_node, int n_elem, int nn, const int *conn, const std::vector<int> &indexL,
                           const std::vector<int> &itemL, const std::vector<int> &indexU,
                           const std::vector<int> &itemU, std::vector<int64_t> &ptr, std::vector<int> &code);

// Block ILU(0) in natural order (FORM_ILU0_33, hecmw_precond_BILU_33.f90:185-362),
// computed on the host from the hecmwST arrays.  Outputs the factor blocks in the
// layout of the input (Dlu0 9N, ALlu0 9NPL, AUlu0 9NPU).  Returns 0 or 9001 on a
// zero pivot.
int factor_bilu0(const Profile &p, const double *D, const double *AL, const double *AU,
                 double sigma_diag, std::vector<double> &Dlu0, std::vector<double> &ALlu0,
                 std::vector<double> &AUlu0);
// The same in place on the D, AL, AU arrays (9 N, 9 NPL, 9 NPU doubles).
int factor_bilu0_inplace(const Profile &p, double *D, double *AL, double *AU, double sigma_diag);

// Fill pattern of the reference's block ILU(1) / ILU(2) (FORM_ILU1_33 / FORM_ILU2_33,
// hecmw_precond_BILU_33.f90:371-739, 748-1337) on the internal rows of p: level-1
// fill = original L(i) x original U(k), not yet in row i; level 2 (ILU(2) only) =
// original L(i) x level-1 U(k) and level-1 L(i) x original U(k).  Each row's lists
// sorted ascending (fill_in_S33_SORT), with the level of every entry and the index
// of its original block (-1 for fill).
struct FilledProfile {
  int N = 0;
  std::vector<int> indexL, itemL, indexU, itemU;  // items 1-based, as hecmwST
  std::vector<int> levL, levU, srcL, srcU;
  Profile view() const { return Profile{N, indexL.data(), itemL.data(), indexU.data(), itemU.data()}; }
};
void bilu_fill(const Profile &p, int level, FilledProfile &f);

// Numeric block ILU(1) / ILU(2) on a filled pattern: D with sigma_diag on its diagonal,
// original values at original positions and zero at fill; row i eliminates with
// every L(i,k) and U(k,j) whose levels sum below `level`, the diagonal included, and
// ends with the reciprocal-pivot LU of its diagonal block.  Returns 0 or 9001 on a
// zero pivot.
int factor_bilu_fill(const FilledProfile &f, int level, const double *D, const double *AL, const double *AU,
                     double sigma_diag, std::vector<double> &Dlu, std::vector<double> &ALlu,
                     std::vector<double> &AUlu);

// Level schedule of the natural-order lower (or upper) triangular solve:
// level[i] = 1 + max level over dependencies.  Rows sorted by group -> order,
// group boundaries in level_ptr.  Lower: group = level (walked first to last).
// Upper: group = maxlevel - level (walked last to first by the backward sweep).
void level_schedule(const Profile &p, bool lower, std::vector<int> &order,
                    std::vector<int> &level_ptr);

// Aggregates of the node graph for the coarse space of the learned two-level
// preconditioner (no counterpart in the reference solver).  One pass: nodes in index
// order; a node whose closed neighbourhood is still free roots a new aggregate of that
// neighbourhood; every node left joins the aggregate of its first neighbour that a
// root took.  The first pass always runs; passes then repeat on the graph of
// aggregates while there are more than max_aggregates and a pass at least halves the
// count, so on a 27-point mesh one pass gives 3x3x3-node aggregates and two give
// 9x9x9.  Also:
//   pptr/pagg: for node i the aggregates of its closed neighbourhood, ascending
//              (the block pattern of the smoothed prolongator's row i);
//   rptr/rnode/rpos: for aggregate a the entries p of pagg with pagg[p] == a, as
//              (node, p) pairs in ascending node order (the restriction's gather).
//   qptr/qagg: for node i the aggregates of its two-ring (the union of pagg over the
//              closed neighbourhood), ascending: the pattern of row i of A P;
//   cptr/cagg: for aggregate a the aggregates b with a nonzero coarse block (a, b),
//              ascending: the union of qagg over the nodes of a's restriction.
struct Aggregation {
  int n_agg = 0;
  std::vector<int> agg;
  std::vector<int> pptr, pagg;
  std::vector<int> rptr, rnode, rpos;
  std::vector<int> qptr, qagg;
  std::vector<int> cptr, cagg;
};
void aggregate_nodes(const Profile &p, int max_aggregates, Aggregation &out);

}  // namespace h33
