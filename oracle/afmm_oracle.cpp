// AFMM2D CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the reference AFMM2D algorithm (vaishna77/AFMM2D)
// used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
// the checker.  The product (afmm2d_b200) never links, imports or executes
// anything in this directory.  Every function cites the reference file:line
// it restates.  Parity of this restatement is pinned against the reference
// itself, compiled here from its own sources (Makefile target "ref"), by the
// CPU tests and by the committed golden fixtures in tests/golden/.
//
// Arithmetic: compiled with -ffp-contract=off (no FMA), like the reference's
// own build flags, so kernel entries and ACA residuals round the same way.
// log/exp and the ACA dot products are correctly rounded (cr_math.h), as in
// the reference build here (its Eigen shim and user kernels) and on the GPU.
// The reference's unqualified abs(double) is taken as the double overload
// (the behaviour its published benchmarks imply).
#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cr_math.h"

namespace {

// ---------------------------------------------------------------- kernels
// Built-in kernels, ids shared with the product.  R2 is formed exactly as in
// examples/testAFMM2D.cpp:12 (dx*dx + dy*dy, no FMA).
struct Kern {
  int id;
  double a;       // smallest box size 2^-L (src/AFMM2DTree.cpp:14-19)
  double param;   // Gaussian width parameter
  double operator()(double xi, double yi, double xj, double yj) const {
    double dx = xi - xj, dy = yi - yj;
    double R2 = dx * dx + dy * dy;
    switch (id) {
      case 0: {  // examples/testAFMM2D.cpp:9-20
        double R = std::sqrt(R2);
        return (R < a) ? R / a : a / R;
      }
      case 1:  // examples/tutorial.cpp:22-35 (log with diagonal convention)
        if (R2 < 1e-10) return 0.0;
        if (R2 < a * a) return 0.5 * R2 * crm::log_cr(R2) / a / a;
        return 0.5 * crm::log_cr(R2);
      case 2:  // 1/r, 0 at r = 0
        if (R2 == 0.0) return 0.0;
        return 1.0 / std::sqrt(R2);
      case 16:  // inverse multiquadric 1/sqrt(R2 + param): the user kernel of the
                // plug-in test (tests/plugin/imq_kernel.cu), registered out of tree
        return 1.0 / std::sqrt(R2 + param);
      default:  // Gaussian exp(-R2/param)
        return crm::exp_cr(-R2 / param);
    }
  }
};

// ------------------------------------------------------------ tree shape
// src/AFMM2D.cpp:7 -- nLevels = log(N/M)/log(4), integer division, truncated.
int n_levels(int N, int M) {
  if (N <= 0 || M <= 0 || N / M < 1) return -1;
  unsigned L = std::log(N / M) / std::log(4);
  return (int)L;
}

// ------------------------------------------------------------ KD sort
// Restatement of src/KDTree.cpp:37-142: rows [x, y, prop]; top-down merge
// sort of a segment by column d in which ties take the RIGHT element first
// (src/KDTree.cpp:47 uses a strict '<').
struct KD {
  std::vector<double> c[3];  // x, y, original index
  std::vector<double> tmp[3];
  int L;
  std::vector<int> counts;

  void merge(unsigned ls, unsigned ln, unsigned rs, unsigned rn, int d) {  // :37-71
    unsigned jl = ls, jr = rs, j = 0;
    for (int k = 0; k < 3; ++k) tmp[k].resize(ln + rn);
    auto take = [&](unsigned src) {
      for (int k = 0; k < 3; ++k) tmp[k][j] = c[k][src];
      ++j;
    };
    while (jl < ls + ln && jr < rs + rn) {
      if (c[d][jl] < c[d][jr]) take(jl++);
      else take(jr++);
    }
    while (jl < ls + ln) take(jl++);
    while (jr < rs + rn) take(jr++);
    for (int k = 0; k < 3; ++k)
      std::copy(tmp[k].begin(), tmp[k].begin() + (ln + rn), c[k].begin() + ls);
  }
  void msort(unsigned s, unsigned n, int d) {  // :73-89
    if (n <= 1) return;
    unsigned ln = n / 2;
    msort(s, ln, d);
    msort(s + ln, n - ln, d);
    merge(s, ln, s + ln, n - ln, d);
  }
  void sort(unsigned s, unsigned n, int d, int level) {  // :91-142
    d %= 2;
    msort(s, n, d);
    unsigned ln = n / 2, rs = s + ln, rn = n - ln;
    d = (d + 1) % 2;
    msort(s, ln, d);
    unsigned lbn = ln / 2, lts = s + lbn, ltn = ln - lbn;
    msort(rs, rn, d);
    unsigned rbn = rn / 2, rts = rs + rbn, rtn = rn - rbn;
    d = (d + 1) % 2;
    if (level < L) {
      ++level;
      if (level == L) {
        counts.push_back((int)lbn);
        counts.push_back((int)ltn);
        counts.push_back((int)rbn);
        counts.push_back((int)rtn);
      }
      sort(s, lbn, d, level);
      sort(lts, ltn, d, level);
      sort(rs, rbn, d, level);
      sort(rts, rtn, d, level);
    }
  }
};

// DFS leaf -> quadtree box number at level L (src/KDTree.cpp:211-223): the
// children of DFS box p are quadtree boxes 4p+0, 4p+3, 4p+1, 4p+2.
std::vector<int> box_numbers(int L) {
  std::vector<int> cur(1, 0);
  for (int j = 1; j <= L; ++j) {
    std::vector<int> nx;
    nx.reserve(cur.size() * 4);
    for (int p : cur) {
      nx.push_back(4 * p + 0);
      nx.push_back(4 * p + 3);
      nx.push_back(4 * p + 1);
      nx.push_back(4 * p + 2);
    }
    cur.swap(nx);
  }
  return cur;
}

// ----------------------------------------------------- interaction lists
// Restatement of the parent-to-child recurrence of src/AFMM2DTree.cpp:65-943
// as a table.  For child c of a box: sibling assignments (neighbour slot,
// child offset from child 0's number) and, for each parent-neighbour slot n
// and each of that neighbour's children g, the (list, slot) it fills.
// List codes: 0 = neighbour, 1 = inner, 2 = outer.
struct Slot { int8_t list, slot; };
const int kSib[4][3][2] = {
    {{3, 1}, {4, 2}, {5, 3}},     // :82-84
    {{7, 0}, {5, 2}, {6, 3}},     // :303-305 (nC-1, nC+1, nC+2 for nC = 4k+1)
    {{0, 0}, {1, 1}, {7, 3}},     // :523-525
    {{1, 0}, {2, 1}, {3, 2}}};    // :743-745
#define N_(s) {0, s}
#define I_(s) {1, s}
#define O_(s) {2, s}
const Slot kRec[4][8][4] = {
    {  // child 0, src/AFMM2DTree.cpp:102-280
     {I_(0), I_(1), N_(0), I_(15)}, {I_(2), I_(3), N_(2), N_(1)},
     {I_(4), O_(7), O_(8), I_(5)},  {I_(6), O_(9), O_(10), I_(7)},
     {I_(8), O_(11), O_(12), O_(13)}, {I_(10), I_(9), O_(14), O_(15)},
     {I_(12), I_(11), O_(16), O_(17)}, {I_(14), N_(7), N_(6), I_(13)}},
    {  // child 1, :323-500
     {O_(23), I_(0), I_(15), O_(22)}, {I_(1), I_(2), N_(1), N_(0)},
     {I_(3), I_(4), I_(5), N_(2)},    {N_(3), I_(6), I_(7), N_(4)},
     {I_(9), I_(8), O_(13), O_(14)},  {I_(11), I_(10), O_(15), O_(16)},
     {O_(19), I_(12), O_(17), O_(18)}, {O_(21), I_(14), I_(13), O_(20)}},
    {  // child 2, :546-720
     {O_(0), O_(1), I_(0), O_(23)},  {O_(2), O_(3), I_(2), I_(1)},
     {O_(4), O_(5), I_(4), I_(3)},   {N_(2), I_(5), I_(6), N_(3)},
     {N_(4), I_(7), I_(8), I_(9)},   {N_(6), N_(5), I_(10), I_(11)},
     {O_(20), I_(13), I_(12), O_(19)}, {O_(22), I_(15), I_(14), O_(21)}},
    {  // child 3, :766-940
     {O_(1), O_(2), I_(1), I_(0)},   {O_(3), O_(4), I_(3), I_(2)},
     {O_(5), O_(6), O_(7), I_(4)},   {I_(5), O_(8), O_(9), I_(6)},
     {I_(7), O_(10), O_(11), I_(8)}, {N_(5), N_(4), I_(9), I_(10)},
     {I_(13), N_(6), I_(11), I_(12)}, {I_(15), N_(0), N_(7), I_(14)}}};
#undef N_
#undef I_
#undef O_

struct Lists {
  // per level: nbr[4^j*8], inner[4^j*16], outer[4^j*24]
  std::vector<std::vector<int>> nbr, inner, outer;
};

// src/AFMM2DTree.cpp:24-62 (createTree) + :947-967 (assign_Tree_Interactions)
Lists lists_recurrence(int L) {
  Lists t;
  t.nbr.resize(L + 1);
  t.inner.resize(L + 1);
  t.outer.resize(L + 1);
  for (int j = 0; j <= L; ++j) {
    size_t nb = (size_t)1 << (2 * j);
    t.nbr[j].assign(nb * 8, -1);
    t.inner[j].assign(nb * 16, -1);
    t.outer[j].assign(nb * 24, -1);
  }
  for (int j = 0; j < L; ++j) {
    size_t nb = (size_t)1 << (2 * j);
    for (size_t k = 0; k < nb; ++k)
      for (int c = 0; c < 4; ++c) {
        int nC = (int)(4 * k + c);
        int* cn = &t.nbr[j + 1][(size_t)nC * 8];
        int* ci = &t.inner[j + 1][(size_t)nC * 16];
        int* co = &t.outer[j + 1][(size_t)nC * 24];
        for (int s = 0; s < 3; ++s) cn[kSib[c][s][0]] = (int)(4 * k) + kSib[c][s][1];
        for (int n = 0; n < 8; ++n) {
          int nN = t.nbr[j][k * 8 + n];
          if (nN == -1) continue;
          for (int g = 0; g < 4; ++g) {
            Slot sl = kRec[c][n][g];
            int child = 4 * nN + g;
            if (sl.list == 0) cn[sl.slot] = child;
            else if (sl.list == 1) ci[sl.slot] = child;
            else co[sl.slot] = child;
          }
        }
      }
  }
  return t;
}

// Closed form of the same lists: box k at level j sits at grid cell (ix, iy)
// given by its base-4 digits (child offsets 0:(0,0) 1:(1,0) 2:(1,1) 3:(0,1),
// src/AFMM2DTree.cpp:978-986).  Slot s of ring m (m = 1 neighbours, 2 inner,
// 3 outer) is the cell at the s-th offset counter-clockwise around the ring
// from (-m,-m); it exists when the cell lies in the domain and, for ring 3,
// when its parent is a neighbour of the box's parent.
void ring_offset(int m, int s, int* dx, int* dy) {
  int side = 2 * m;
  int x = -m, y = -m;
  int seg = s / side, t = s % side;
  if (seg == 0) { x = -m + t; y = -m; }
  else if (seg == 1) { x = m; y = -m + t; }
  else if (seg == 2) { x = m - t; y = m; }
  else { x = -m; y = m - t; }
  *dx = x;
  *dy = y;
}
void cell_of(long k, int j, int* ix, int* iy) {
  static const int ox[4] = {0, 1, 1, 0}, oy[4] = {0, 0, 1, 1};
  int x = 0, y = 0;
  for (int l = j - 1; l >= 0; --l) {
    int d = (int)((k >> (2 * l)) & 3);
    x = 2 * x + ox[d];
    y = 2 * y + oy[d];
  }
  *ix = x;
  *iy = y;
}
long box_of(int ix, int iy, int j) {
  long k = 0;
  for (int l = j - 1; l >= 0; --l) {
    int bx = (ix >> l) & 1, by = (iy >> l) & 1;
    int d = by ? (bx ? 2 : 3) : (bx ? 1 : 0);
    k = 4 * k + d;
  }
  return k;
}
void lists_closed_form(int j, int* nbr, int* inner, int* outer) {
  long nb = 1L << (2 * j);
  int side = 1 << j;
  for (long k = 0; k < nb; ++k) {
    int ix, iy;
    cell_of(k, j, &ix, &iy);
    for (int m = 1; m <= 3; ++m) {
      int ns = 8 * m;
      int* out = (m == 1) ? nbr + k * 8 : (m == 2) ? inner + k * 16 : outer + k * 24;
      for (int s = 0; s < ns; ++s) {
        int dx, dy;
        ring_offset(m, s, &dx, &dy);
        int cx = ix + dx, cy = iy + dy;
        bool ok = cx >= 0 && cy >= 0 && cx < side && cy < side;
        if (ok && m == 3) ok = std::abs((cx >> 1) - (ix >> 1)) <= 1 && std::abs((cy >> 1) - (iy >> 1)) <= 1;
        out[s] = ok ? (int)box_of(cx, cy, j) : -1;
      }
    }
  }
}

// ---------------------------------------------------------------- tree
struct Box {
  std::vector<int> nodes;       // incoming check points of children / points
  std::vector<int> skel;        // incoming_checkPoints
  std::vector<int> cpts;        // incoming_chargePoints
  std::vector<double> l2p;      // n x r, row-major
  int n = 0, r = 0;
  std::vector<double> out, in;  // outgoing_charges, incoming_potential
  std::vector<double> pot;      // leaf potential
};

struct Oracle {
  int N, M, tol_pow, L, status;
  Kern K;
  std::vector<double> xy;      // sorted locations, interleaved
  std::vector<int64_t> perm;   // sorted i -> original index
  std::vector<int> counts, boxnum;
  std::vector<int> leaf_start; // by quadtree leaf number
  Lists lists;
  std::vector<std::vector<Box>> tree;
  // M2L[j][k] : map slot-order list of (c, matrix r_k x r_c row-major)
  std::vector<std::vector<std::vector<std::pair<int, std::vector<double>>>>> m2l;

  double k(int i, int j) const { return K(xy[2 * i], xy[2 * i + 1], xy[2 * j], xy[2 * j + 1]); }
};

// src/ACA.cpp:12-25 -- first maximal |v| over the allowed set in ascending order.
int argmax_abs(const std::vector<double>& v, const std::vector<char>& allowed) {
  int idx = -1;
  double mx = 0;
  for (size_t i = 0; i < v.size(); ++i) {
    if (!allowed[i]) continue;
    if (idx < 0) { idx = (int)i; mx = std::fabs(v[i]); continue; }
    if (std::fabs(v[i]) > mx) { idx = (int)i; mx = std::fabs(v[i]); }
  }
  return idx < 0 ? 0 : idx;  // an empty set yields index 0 (never used)
}

// Correctly rounded dot product (the shim's VectorXd::dot and squaredNorm).
double dotp(const std::vector<double>& a, const std::vector<double>& b) {
  return crm::dot_cr(a.data(), b.data(), (long)a.size());
}

// src/ACA.cpp:27-133 -- partially pivoted ACA returning row/col pivots.
void aca(const Oracle& o, const std::vector<int>& rows, const std::vector<int>& cols, double tol,
         std::vector<int>& rb, std::vector<int>& cb) {
  int n1 = (int)rows.size(), n2 = (int)cols.size();
  int mn = std::min(n1, n2);
  if (mn == 0) return;  // no rows or no columns: rank 0
  std::vector<std::vector<double>> U, V;
  std::vector<char> rrem(n1, 1), crem(n2, 1);
  std::vector<double> row(n2), col(n1), v(n2);
  auto get_row = [&](int ri) { for (int s = 0; s < n2; ++s) row[s] = o.k(rows[ri], cols[s]); };
  auto get_col = [&](int cj) { for (int i = 0; i < n1; ++i) col[i] = o.k(rows[i], cols[cj]); };
  int ri = 0, cj = 0, l;
  for (l = 0; l < n1; ++l) {  // :56-63
    ri = l;
    get_row(ri);
    cj = argmax_abs(row, crem);
    if (std::fabs(row[cj]) > tol) break;
  }
  if (l == n1) return;  // rank 0, :64-68
  for (int s = 0; s < n2; ++s) v[s] = row[s] / row[cj];
  rb.push_back(ri);
  cb.push_back(cj);
  get_col(cj);
  U.push_back(col);
  V.push_back(v);
  crem[cj] = 0;
  rrem[ri] = 0;
  int rank = 1;
  double normS = 0.0, prev = DBL_MAX;
  ri = argmax_abs(col, rrem);  // :84
  while (std::fabs(prev - normS) >= tol * prev && rank < mn) {  // :86
    rb.push_back(ri);
    get_row(ri);
    for (int q = 0; q < rank; ++q)
      for (int s = 0; s < n2; ++s) row[s] -= U[q][ri] * V[q][s];
    cj = argmax_abs(row, crem);
    cb.push_back(cj);
    for (int s = 0; s < n2; ++s) v[s] = row[s] / row[cj];
    get_col(cj);
    for (int q = 0; q < rank; ++q)
      for (int i = 0; i < n1; ++i) col[i] -= V[q][cj] * U[q][i];
    U.push_back(col);
    V.push_back(v);
    ++rank;
    crem[cj] = 0;
    rrem[ri] = 0;
    if (rank != 2) prev = normS;  // :122-123
    double un = std::sqrt(dotp(col, col)), vn = std::sqrt(dotp(v, v));
    normS = std::pow(normS, 2) + std::pow(un * vn, 2);  // :124
    for (int q = 0; q < rank; ++q) normS += 2 * std::fabs(dotp(U[q], col) * dotp(V[q], v));
    normS = std::sqrt(normS);
    ri = argmax_abs(col, rrem);  // :129
  }
}

// Solve X D = A for X (n x r) with D = K(R, C), via LU of D^T with partial
// pivoting (src/AFMM2DTree.cpp:1057-1059).
std::vector<double> l2p_solve(const std::vector<double>& D, const std::vector<double>& Ac, int n, int r) {
  // A = D^T (r x r), B = Ac^T (r x n); solve A X' = B, X = X'^T.
  std::vector<double> A(r * r);
  for (int i = 0; i < r; ++i)
    for (int j = 0; j < r; ++j) A[i * r + j] = D[j * r + i];
  std::vector<int> p(r);
  for (int i = 0; i < r; ++i) p[i] = i;
  for (int kk = 0; kk < r; ++kk) {
    int piv = kk;
    double best = std::fabs(A[kk * r + kk]);
    for (int i = kk + 1; i < r; ++i)
      if (std::fabs(A[i * r + kk]) > best) { best = std::fabs(A[i * r + kk]); piv = i; }
    if (piv != kk) {
      for (int j = 0; j < r; ++j) std::swap(A[kk * r + j], A[piv * r + j]);
      std::swap(p[kk], p[piv]);
    }
    double d = A[kk * r + kk];
    if (d != 0.0)
      for (int i = kk + 1; i < r; ++i) {
        double f = A[i * r + kk] / d;
        A[i * r + kk] = f;
        for (int j = kk + 1; j < r; ++j) A[i * r + j] -= f * A[kk * r + j];
      }
  }
  std::vector<double> X(n * r);
  std::vector<double> x(r);
  for (int c = 0; c < n; ++c) {
    for (int i = 0; i < r; ++i) {
      double s = Ac[c * r + p[i]];
      for (int j = 0; j < i; ++j) s -= A[i * r + j] * x[j];
      x[i] = s;
    }
    for (int i = r - 1; i >= 0; --i) {
      double s = x[i];
      for (int j = i + 1; j < r; ++j) s -= A[i * r + j] * x[j];
      x[i] = s / A[i * r + i];
    }
    for (int i = 0; i < r; ++i) X[c * r + i] = x[i];
  }
  return X;
}

// src/AFMM2DTree.cpp:997-1007 -- a non-leaf box's nodes are its children's
// skeletons, children 0..3 in order.
void build_nodes(Oracle& o, int j) {
  for (size_t k = 0; k < o.tree[j].size(); ++k) {
    Box& b = o.tree[j][k];
    if (j == o.L) continue;  // leaves set in create
    b.nodes.clear();
    for (int c = 0; c < 4; ++c) {
      const Box& ch = o.tree[j + 1][4 * k + c];
      b.nodes.insert(b.nodes.end(), ch.skel.begin(), ch.skel.end());
    }
  }
}

// src/AFMM2DTree.cpp:1009-1061
void assemble_box(Oracle& o, int j, int k, double tol) {
  Box& b = o.tree[j][k];
  const std::vector<int>& rows = b.nodes;
  std::vector<int> cols;
  for (int in = 0; in < 16; ++in) {
    int c = o.lists.inner[j][(size_t)k * 16 + in];
    if (c != -1) cols.insert(cols.end(), o.tree[j][c].nodes.begin(), o.tree[j][c].nodes.end());
  }
  for (int on = 0; on < 24; ++on) {
    int c = o.lists.outer[j][(size_t)k * 24 + on];
    if (c != -1) cols.insert(cols.end(), o.tree[j][c].nodes.begin(), o.tree[j][c].nodes.end());
  }
  std::vector<int> rb, cb;
  aca(o, rows, cols, tol, rb, cb);
  int r = (int)rb.size(), n = (int)rows.size();
  b.n = n;
  b.r = r;
  b.skel.clear();
  b.cpts.clear();
  b.l2p.clear();
  if (r == 0) return;
  for (int q = 0; q < r; ++q) b.skel.push_back(rows[rb[q]]);
  for (int q = 0; q < r; ++q) b.cpts.push_back(cols[cb[q]]);
  std::vector<double> D(r * r), Ac(n * r);
  for (int i = 0; i < r; ++i)
    for (int q = 0; q < r; ++q) D[i * r + q] = o.k(b.skel[i], b.cpts[q]);
  for (int i = 0; i < n; ++i)
    for (int q = 0; q < r; ++q) Ac[i * r + q] = o.k(rows[i], b.cpts[q]);
  b.l2p = l2p_solve(D, Ac, n, r);
}

}  // namespace

extern "C" {

int afo_nlevels(int N, int M) { return n_levels(N, M); }

// xy: N points interleaved.  Returns NULL when nLevels < 2 (the reference
// crashes there: src/AFMM2DTree.cpp:1207 with an empty leaf potential).
void* afo_create(int N, int M, int tol_pow, const double* xy, int kernel_id, double kparam) {
  int L = n_levels(N, M);
  if (L < 2) return nullptr;
  Oracle* o = new Oracle();
  o->N = N;
  o->M = M;
  o->tol_pow = tol_pow;
  o->L = L;
  o->status = 0;
  o->K = Kern{kernel_id, std::pow(0.5, L), kparam};
  // src/AFMM2DTree.cpp:14-19: a = boxRadius[L] with boxRadius halving from 1.
  double a = 1.0;
  for (int j = 0; j < L; ++j) a *= 0.5;
  o->K.a = a;
  KD kd;
  kd.L = L;
  for (int k = 0; k < 3; ++k) kd.c[k].resize(N);
  for (int i = 0; i < N; ++i) {  // src/AFMM2D.cpp:16-25
    kd.c[0][i] = xy[2 * i];
    kd.c[1][i] = xy[2 * i + 1];
    kd.c[2][i] = i;
  }
  if (N > 1) kd.sort(0, N, 0, 0);  // src/KDTree.cpp:144-153
  o->xy.resize(2 * (size_t)N);
  o->perm.resize(N);
  for (int i = 0; i < N; ++i) {
    o->xy[2 * i] = kd.c[0][i];
    o->xy[2 * i + 1] = kd.c[1][i];
    o->perm[i] = (int64_t)kd.c[2][i];
  }
  o->counts = kd.counts;
  o->boxnum = box_numbers(L);
  o->lists = lists_recurrence(L);
  o->tree.resize(L + 1);
  for (int j = 0; j <= L; ++j) o->tree[j].resize((size_t)1 << (2 * j));
  // src/AFMM2DTree.cpp:1099-1118: leaf boxNumbers[k] owns a contiguous range.
  o->leaf_start.assign(o->boxnum.size(), 0);
  int start = 0;
  for (size_t k = 0; k < o->boxnum.size(); ++k) {
    Box& b = o->tree[L][o->boxnum[k]];
    o->leaf_start[o->boxnum[k]] = start;
    b.nodes.resize(o->counts[k]);
    for (int i = 0; i < o->counts[k]; ++i) b.nodes[i] = start + i;
    start += o->counts[k];
  }
  return o;
}

void afo_destroy(void* h) { delete (Oracle*)h; }

// src/AFMM2DTree.cpp:991-995 + :1063-1068 (getNodes), :1070-1097 (assemble_M2L)
void afo_assemble(void* h) {
  Oracle* o = (Oracle*)h;
  double tol = std::pow(10, -1.0 * o->tol_pow);  // src/ACA.cpp:7
  for (int j = o->L; j >= 2; --j) {
    build_nodes(*o, j);
    int nb = (int)o->tree[j].size();
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < nb; ++k) assemble_box(*o, j, k, tol);
  }
  o->m2l.assign(o->L + 1, {});
  for (int j = 2; j <= o->L; ++j) {
    int nb = (int)o->tree[j].size();
    o->m2l[j].resize(nb);
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < nb; ++k) {
      const Box& b = o->tree[j][k];
      for (int s = 0; s < 40; ++s) {
        int c = s < 16 ? o->lists.inner[j][(size_t)k * 16 + s] : o->lists.outer[j][(size_t)k * 24 + s - 16];
        if (c == -1) continue;
        const Box& bc = o->tree[j][c];
        std::vector<double> m((size_t)b.r * bc.r);
        for (int i = 0; i < b.r; ++i)
          for (int q = 0; q < bc.r; ++q) m[(size_t)i * bc.r + q] = o->k(b.skel[i], bc.skel[q]);
        o->m2l[j][k].push_back({c, std::move(m)});
      }
    }
  }
}

// src/AFMM2D.cpp:46-65 and src/AFMM2DTree.cpp:1120-1225.  A rank-0 box
// contributes no far field (the reference aborts on it instead).
void afo_matvec(void* h, const double* q, double* y) {
  Oracle* o = (Oracle*)h;
  int L = o->L, N = o->N;
  std::vector<double> qs(N);
  for (int i = 0; i < N; ++i) qs[i] = q[o->perm[i]];  // :49-51
  // M2M, src/AFMM2DTree.cpp:1129-1154
  for (int j = L; j >= 2; --j) {
    int nb = (int)o->tree[j].size();
#pragma omp parallel for
    for (int k = 0; k < nb; ++k) {
      Box& b = o->tree[j][k];
      std::vector<double> src;
      if (j == L) src.assign(qs.begin() + o->leaf_start[k], qs.begin() + o->leaf_start[k] + b.nodes.size());
      else
        for (int c = 0; c < 4; ++c) {
          const Box& ch = o->tree[j + 1][4 * k + c];
          src.insert(src.end(), ch.out.begin(), ch.out.end());
        }
      b.out.assign(b.r, 0.0);
      for (int i = 0; i < b.n; ++i)
        for (int c = 0; c < b.r; ++c) b.out[c] += b.l2p[(size_t)i * b.r + c] * src[i];
    }
  }
  // M2L, :1156-1178 (slot order inner 0..15 then outer 0..23)
  for (int j = 2; j <= L; ++j) {
    int nb = (int)o->tree[j].size();
#pragma omp parallel for
    for (int k = 0; k < nb; ++k) {
      Box& b = o->tree[j][k];
      b.in.assign(b.r, 0.0);
      for (auto& pr : o->m2l[j][k]) {
        const Box& bc = o->tree[j][pr.first];
        std::vector<double> t(b.r, 0.0);
        for (int q2 = 0; q2 < bc.r; ++q2)
          for (int i = 0; i < b.r; ++i) t[i] += pr.second[(size_t)i * bc.r + q2] * bc.out[q2];
        for (int i = 0; i < b.r; ++i) b.in[i] += t[i];
      }
    }
  }
  // L2L, :1180-1197
  for (int j = 2; j <= L; ++j) {
    int nb = (int)o->tree[j].size();
#pragma omp parallel for
    for (int k = 0; k < nb; ++k) {
      Box& b = o->tree[j][k];
      std::vector<double> t(b.n, 0.0);
      for (int c = 0; c < b.r; ++c)
        for (int i = 0; i < b.n; ++i) t[i] += b.l2p[(size_t)i * b.r + c] * b.in[c];
      if (j != L) {
        int off = 0;
        for (int c = 0; c < 4; ++c) {
          Box& ch = o->tree[j + 1][4 * k + c];
          for (int i = 0; i < ch.r; ++i) ch.in[i] += t[off + i];
          off += ch.r;
        }
      } else {
        b.pot = t;
      }
    }
  }
  // Near field, :1199-1213 (neighbours 0..7, then self)
  int nl = (int)o->tree[L].size();
#pragma omp parallel for
  for (int k = 0; k < nl; ++k) {
    Box& b = o->tree[L][k];
    int ni = (int)b.nodes.size();
    if ((int)b.pot.size() != ni) b.pot.assign(ni, 0.0);
    for (int n = 0; n <= 8; ++n) {
      int nn = n < 8 ? o->lists.nbr[L][(size_t)k * 8 + n] : k;
      if (nn == -1) continue;
      const Box& bn = o->tree[L][nn];
      int s0 = o->leaf_start[nn];
      std::vector<double> t(ni, 0.0);
      for (size_t q2 = 0; q2 < bn.nodes.size(); ++q2)
        for (int i = 0; i < ni; ++i) t[i] += o->k(b.nodes[i], s0 + (int)q2) * qs[s0 + q2];
      for (int i = 0; i < ni; ++i) b.pot[i] += t[i];
    }
  }
  // :1215-1225 and src/AFMM2D.cpp:61-63
  for (int k = 0; k < nl; ++k) {
    const Box& b = o->tree[L][k];
    int s0 = o->leaf_start[k];
    for (size_t i = 0; i < b.pot.size(); ++i) y[o->perm[s0 + i]] = b.pot[i];
  }
}

int afo_get_nlevels(void* h) { return ((Oracle*)h)->L; }

void afo_get_permutation(void* h, int64_t* perm) {
  Oracle* o = (Oracle*)h;
  std::memcpy(perm, o->perm.data(), sizeof(int64_t) * o->N);
}

void afo_get_sorted_locations(void* h, double* xy) {
  Oracle* o = (Oracle*)h;
  std::memcpy(xy, o->xy.data(), sizeof(double) * 2 * o->N);
}

void afo_get_leaves(void* h, int32_t* counts, int32_t* box_numbers_out) {
  Oracle* o = (Oracle*)h;
  for (size_t k = 0; k < o->counts.size(); ++k) {
    counts[k] = o->counts[k];
    box_numbers_out[k] = o->boxnum[k];
  }
}

void afo_get_lists(void* h, int level, int32_t* nbr, int32_t* inner, int32_t* outer) {
  Oracle* o = (Oracle*)h;
  size_t nb = (size_t)1 << (2 * level);
  for (size_t i = 0; i < nb * 8; ++i) nbr[i] = o->lists.nbr[level][i];
  for (size_t i = 0; i < nb * 16; ++i) inner[i] = o->lists.inner[level][i];
  for (size_t i = 0; i < nb * 24; ++i) outer[i] = o->lists.outer[level][i];
}

// Lists of one level from the closed form (no tree needed).
void afo_lists_closed_form(int level, int32_t* nbr, int32_t* inner, int32_t* outer) {
  lists_closed_form(level, nbr, inner, outer);
}

void afo_get_ranks(void* h, int level, int32_t* ranks) {
  Oracle* o = (Oracle*)h;
  for (size_t k = 0; k < o->tree[level].size(); ++k) ranks[k] = o->tree[level][k].r;
}

long afo_get_skeletons(void* h, int level, int32_t* ids) {
  Oracle* o = (Oracle*)h;
  long c = 0;
  for (auto& b : o->tree[level])
    for (int id : b.skel) {
      if (ids) ids[c] = id;
      ++c;
    }
  return c;
}

long afo_get_charge_points(void* h, int level, int32_t* ids) {
  Oracle* o = (Oracle*)h;
  long c = 0;
  for (auto& b : o->tree[level])
    for (int id : b.cpts) {
      if (ids) ids[c] = id;
      ++c;
    }
  return c;
}

long afo_get_l2p(void* h, int level, int k, int32_t* rows, int32_t* cols, double* out) {
  Oracle* o = (Oracle*)h;
  const Box& b = o->tree[level][k];
  *rows = b.r ? b.n : 0;
  *cols = b.r;
  if (out && b.r) std::memcpy(out, b.l2p.data(), sizeof(double) * b.l2p.size());
  return (long)b.l2p.size();
}

long afo_get_stage(void* h, int level, int which, double* out) {
  Oracle* o = (Oracle*)h;
  long c = 0;
  for (auto& b : o->tree[level]) {
    const std::vector<double>& v = which == 0 ? b.out : b.in;
    for (double x : v) {
      if (out) out[c] = x;
      ++c;
    }
  }
  return c;
}

// Dense FP64 matvec over selected rows, in the original point order:
// y[t] = sum_j K(x_rows[t], x_j) q_j, summed with Neumaier compensation.
// `a` is the kernel's box-size parameter 2^-L.
void afo_dense_rows(int N, const double* xy, int kernel_id, double a, double kparam, const double* q,
                    int nrows, const int64_t* rows, double* y) {
  Kern K{kernel_id, a, kparam};
#pragma omp parallel for schedule(dynamic, 8)
  for (int t = 0; t < nrows; ++t) {
    int64_t i = rows[t];
    double s = 0.0, c = 0.0;
    for (int j = 0; j < N; ++j) {
      double v = K(xy[2 * i], xy[2 * i + 1], xy[2 * j], xy[2 * j + 1]) * q[j];
      double tt = s + v;
      if (std::fabs(s) >= std::fabs(v)) c += (s - tt) + v;
      else c += (v - tt) + s;
      s = tt;
    }
    y[t] = s + c;
  }
}

// The KD permutation through the equivalent total-order formulation (no
// merge sort): every x-sort at level >= 1 orders by (x asc, y desc, index
// desc), the level-0 x-sort by (x asc, index desc), and every y-sort by
// (y asc, x desc, index asc).  Used to cross-check that formulation.
void afo_kd_total_order(int N, int L, const double* xy, int64_t* perm) {
  std::vector<int> p(N);
  for (int i = 0; i < N; ++i) p[i] = i;
  auto X = [&](int i) { return xy[2 * i]; };
  auto Y = [&](int i) { return xy[2 * i + 1]; };
  auto kx0 = [&](int a, int b) { return X(a) < X(b) || (X(a) == X(b) && a > b); };
  auto kx = [&](int a, int b) {
    if (X(a) != X(b)) return X(a) < X(b);
    if (Y(a) != Y(b)) return Y(a) > Y(b);
    return a > b;
  };
  auto ky = [&](int a, int b) {
    if (Y(a) != Y(b)) return Y(a) < Y(b);
    if (X(a) != X(b)) return X(a) > X(b);
    return a < b;
  };
  struct Seg { int s, n, level; };
  std::vector<Seg> st{{0, N, 0}};
  while (!st.empty()) {
    Seg g = st.back();
    st.pop_back();
    if (g.n <= 1 && g.level >= L) continue;
    auto b = p.begin() + g.s;
    if (g.level == 0) std::sort(b, b + g.n, kx0);
    else std::sort(b, b + g.n, kx);
    int ln = g.n / 2, rn = g.n - ln;
    std::sort(b, b + ln, ky);
    std::sort(b + ln, b + g.n, ky);
    if (g.level < L) {
      int lb = ln / 2, rb = rn / 2;
      st.push_back({g.s + ln + rb, rn - rb, g.level + 1});
      st.push_back({g.s + ln, rb, g.level + 1});
      st.push_back({g.s + lb, ln - lb, g.level + 1});
      st.push_back({g.s, lb, g.level + 1});
    }
  }
  for (int i = 0; i < N; ++i) perm[i] = p[i];
}

// K(xy1[t], xy2[t]) with the restated kernels (host libm).
void afo_kernel_pairs(int kernel_id, double a, double param, long n, const double* xy1, const double* xy2,
                      double* out) {
  Kern K{kernel_id, a, param};
  for (long t = 0; t < n; ++t) out[t] = K(xy1[2 * t], xy1[2 * t + 1], xy2[2 * t], xy2[2 * t + 1]);
}

int afo_num_threads(void) { return omp_get_max_threads(); }
}
