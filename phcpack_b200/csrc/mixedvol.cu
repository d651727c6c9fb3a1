// mixedvol.cu -- the mixed volume of the Newton polytopes of a square
// polynomial system (the BKK root count), host code only (no device work):
// the feeder of a start system with one path per root.
//
// The method of MixedVol (Gao, Li and Wu, ACM TOMS 31(4):555-560, 2005;
// Root_Counts/MixedVol/mixedvol_algorithm.adb, mixed_volume1.c,
// relation_table1.c, one_level_lp1.c): every support point gets a random
// lifting value w; a mixed cell is a choice of one edge {a_i, b_i} from
// every support such that one inner normal (alpha, 1) makes all of them
// lower edges, <a_i, alpha> + w(a_i) = <b_i, alpha> + w(b_i) <= <c, alpha>
// + w(c) for every point c of support i; the mixed volume is the sum of
// |det(b_i - a_i)| over the mixed cells.  The search: the lower edges of
// every support alone, the table of pairs of edges of two supports that
// share a normal, and a depth-first search over the supports (fewest lower
// edges first) that extends a choice only by an edge related to every edge
// chosen so far and keeps it while its system of constraints is feasible;
// at the last support the normal solves the n equalities and is checked
// directly.
//
// Feasibility of {alpha : E alpha = f, U alpha <= g}: the equalities are
// eliminated (alpha = alpha_0 + N beta, Gaussian elimination with partial
// pivoting), and M beta <= h is decided through its Farkas dual:
// infeasible exactly when some y >= 0 has M^T y = 0 and h^T y < 0, i.e.
// when min h^T y over {M^T y = 0, sum y = 1, y >= 0} is negative; that LP
// has d + 1 rows (d <= n free directions), solved by a two-phase dense
// simplex with Bland's rule.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "../../include/phc_b200.h"

namespace {

const double kTol = 1e-9;

// min c^T y subject to A y = b (rows x cols, b >= 0), y >= 0; two phases,
// Bland's rule.  Returns 0 with *val set, 1 when infeasible, 2 when
// unbounded (cannot happen for the Farkas dual, whose y lie in a simplex).
int simplex_min(int rows, int cols, const std::vector<double> &A, const std::vector<double> &b,
                const std::vector<double> &c, double *val) {
  const int W = cols + rows + 1;  // y, artificials, right-hand side
  std::vector<double> T((size_t)(rows + 1) * W, 0.0);
  std::vector<int> basis(rows);
  for (int r = 0; r < rows; ++r) {
    for (int j = 0; j < cols; ++j) T[(size_t)r * W + j] = A[(size_t)r * cols + j];
    T[(size_t)r * W + cols + r] = 1.0;
    T[(size_t)r * W + W - 1] = b[r];
    basis[r] = cols + r;
  }
  auto pivot = [&](int pr, int pc) {
    const double p = T[(size_t)pr * W + pc];
    for (int j = 0; j < W; ++j) T[(size_t)pr * W + j] /= p;
    for (int r = 0; r <= rows; ++r) {
      if (r == pr) continue;
      const double f = T[(size_t)r * W + pc];
      if (f == 0.0) continue;
      for (int j = 0; j < W; ++j) T[(size_t)r * W + j] -= f * T[(size_t)pr * W + j];
    }
    basis[pr] = pc;
  };
  // objective row (last): reduced costs; phase 1 minimises the artificials
  auto set_objective = [&](bool phase1) {
    double *z = &T[(size_t)rows * W];
    std::fill(z, z + W, 0.0);
    for (int j = 0; j < cols; ++j) z[j] = phase1 ? 0.0 : c[j];
    if (phase1)
      for (int r = 0; r < rows; ++r) z[cols + r] = 1.0;
    for (int r = 0; r < rows; ++r) {
      const double cb = basis[r] >= cols ? (phase1 ? 1.0 : 0.0) : (phase1 ? 0.0 : c[basis[r]]);
      if (cb == 0.0) continue;
      for (int j = 0; j < W; ++j) z[j] -= cb * T[(size_t)r * W + j];
    }
  };
  auto run = [&](int ncols_allowed) -> int {
    for (int it = 0; it < 50000; ++it) {
      int pc = -1;
      for (int j = 0; j < ncols_allowed; ++j)
        if (T[(size_t)rows * W + j] < -kTol) { pc = j; break; }  // Bland: the first improving column
      if (pc < 0) return 0;
      int pr = -1;
      double best = 0.0;
      for (int r = 0; r < rows; ++r) {
        const double a = T[(size_t)r * W + pc];
        if (a > kTol) {
          const double q = T[(size_t)r * W + W - 1] / a;
          if (pr < 0 || q < best - 1e-15 || (std::fabs(q - best) <= 1e-15 && basis[r] < basis[pr])) {
            pr = r;
            best = q;
          }
        }
      }
      if (pr < 0) return 2;
      pivot(pr, pc);
    }
    return 3;
  };
  set_objective(true);
  if (run(cols + rows) != 0) return 1;
  if (-T[(size_t)rows * W + W - 1] > 1e-9) return 1;
  // drive the artificials out of the basis where a column allows it
  for (int r = 0; r < rows; ++r)
    if (basis[r] >= cols)
      for (int j = 0; j < cols; ++j)
        if (std::fabs(T[(size_t)r * W + j]) > kTol) { pivot(r, j); break; }
  set_objective(false);
  const int rc = run(cols);
  if (rc != 0) return rc;
  *val = -T[(size_t)rows * W + W - 1];
  return 0;
}

// Is {alpha : E alpha = f, U alpha <= g} nonempty?  E: k x n, U: m x n.
bool feasible(int n, const std::vector<double> &E, const std::vector<double> &f, const std::vector<double> &U,
              const std::vector<double> &g) {
  const int k = (int)f.size(), m = (int)g.size();
  // row echelon form of [E | f]: pivot columns, and alpha = a0 + N beta
  std::vector<double> R(E), rf(f);
  std::vector<int> pcol;
  int row = 0;
  std::vector<char> is_piv(n, 0);
  for (int col = 0; col < n && row < k; ++col) {
    int best = -1;
    double bv = kTol;
    for (int r = row; r < k; ++r)
      if (std::fabs(R[(size_t)r * n + col]) > bv) { bv = std::fabs(R[(size_t)r * n + col]); best = r; }
    if (best < 0) continue;
    for (int j = 0; j < n; ++j) std::swap(R[(size_t)row * n + j], R[(size_t)best * n + j]);
    std::swap(rf[row], rf[best]);
    const double p = R[(size_t)row * n + col];
    for (int j = 0; j < n; ++j) R[(size_t)row * n + j] /= p;
    rf[row] /= p;
    for (int r = 0; r < k; ++r) {
      if (r == row) continue;
      const double q = R[(size_t)r * n + col];
      if (q == 0.0) continue;
      for (int j = 0; j < n; ++j) R[(size_t)r * n + j] -= q * R[(size_t)row * n + j];
      rf[r] -= q * rf[row];
    }
    pcol.push_back(col);
    is_piv[col] = 1;
    ++row;
  }
  for (int r = row; r < k; ++r)
    if (std::fabs(rf[r]) > 1e-8) return false;  // inconsistent equalities
  std::vector<int> freec;
  for (int j = 0; j < n; ++j)
    if (!is_piv[j]) freec.push_back(j);
  const int d = (int)freec.size();
  // alpha = a0 + N beta: pivot variable of row r = rf[r] - sum_free R[r][j] beta_j
  std::vector<double> a0(n, 0.0), N((size_t)n * (d > 0 ? d : 1), 0.0);
  for (int r = 0; r < row; ++r) {
    a0[pcol[r]] = rf[r];
    for (int q = 0; q < d; ++q) N[(size_t)pcol[r] * d + q] = -R[(size_t)r * n + freec[q]];
  }
  for (int q = 0; q < d; ++q) N[(size_t)freec[q] * d + q] = 1.0;
  // M beta <= h with M = U N, h = g - U a0
  std::vector<double> M((size_t)m * (d > 0 ? d : 1), 0.0), h(m);
  for (int i = 0; i < m; ++i) {
    double s = g[i];
    for (int j = 0; j < n; ++j) s -= U[(size_t)i * n + j] * a0[j];
    h[i] = s;
    for (int q = 0; q < d; ++q) {
      double v = 0.0;
      for (int j = 0; j < n; ++j) v += U[(size_t)i * n + j] * N[(size_t)j * d + q];
      M[(size_t)i * d + q] = v;
    }
  }
  if (d == 0) {
    for (int i = 0; i < m; ++i)
      if (h[i] < -1e-9) return false;
    return true;
  }
  if (m == 0) return true;
  // the Farkas dual: rows M^T y = 0 (d) and sum y = 1
  std::vector<double> A((size_t)(d + 1) * m), b(d + 1, 0.0);
  for (int q = 0; q < d; ++q)
    for (int i = 0; i < m; ++i) A[(size_t)q * m + i] = M[(size_t)i * d + q];
  for (int i = 0; i < m; ++i) A[(size_t)d * m + i] = 1.0;
  b[d] = 1.0;
  double val = 0.0;
  const int rc = simplex_min(d + 1, m, A, b, h, &val);
  if (rc == 1) return true;  // no y: by Gordan, M beta < 0 has a solution
  if (rc != 0) return true;  // not decided: keep the branch (the leaves are checked exactly)
  return val >= -1e-9;
}

struct Edge {
  int p, q;
};

struct Search {
  int n;
  std::vector<std::vector<std::vector<int> > > pts;  // pts[i][c][j]
  std::vector<std::vector<double> > w;
  std::vector<std::vector<Edge> > edges;
  std::vector<int> order;
  std::vector<std::vector<char> > rel;  // rel[a*n+b][e*|E_b|+f] for a < b in search order
  long long mv = 0;
  long long ncells = 0;
  int max_cells = 0;
  int *cells = nullptr;

  // the rows of edge e of support i: equality and inequalities
  void rows(int i, const Edge &e, std::vector<double> &E, std::vector<double> &f, std::vector<double> &U,
            std::vector<double> &g) const {
    const auto &P = pts[i];
    for (int j = 0; j < n; ++j) E.push_back((double)(P[e.q][j] - P[e.p][j]));
    f.push_back(w[i][e.p] - w[i][e.q]);
    for (size_t c = 0; c < P.size(); ++c) {
      for (int j = 0; j < n; ++j) U.push_back(-(double)(P[c][j] - P[e.p][j]));
      g.push_back(w[i][c] - w[i][e.p]);
    }
  }

  bool feasible_choice(const std::vector<int> &sup, const std::vector<Edge> &ch) const {
    std::vector<double> E, f, U, g;
    for (size_t k = 0; k < ch.size(); ++k) rows(sup[k], ch[k], E, f, U, g);
    return feasible(n, E, f, U, g);
  }

  void leaf(const std::vector<Edge> &ch) {
    // alpha from the n equalities, then every inequality
    std::vector<double> D((size_t)n * n), r(n);
    for (int k = 0; k < n; ++k) {
      const int i = order[k];
      for (int j = 0; j < n; ++j) D[(size_t)k * n + j] = (double)(pts[i][ch[k].q][j] - pts[i][ch[k].p][j]);
      r[k] = w[i][ch[k].p] - w[i][ch[k].q];
    }
    // the volume |det D| (integers) and the solve, by partial pivoting
    std::vector<double> LU(D);
    std::vector<double> x(r);
    double det = 1.0;
    for (int c = 0; c < n; ++c) {
      int pr = c;
      for (int q = c + 1; q < n; ++q)
        if (std::fabs(LU[(size_t)q * n + c]) > std::fabs(LU[(size_t)pr * n + c])) pr = q;
      if (std::fabs(LU[(size_t)pr * n + c]) < 1e-12) return;  // dependent edges: no cell
      if (pr != c) {
        for (int j = 0; j < n; ++j) std::swap(LU[(size_t)pr * n + j], LU[(size_t)c * n + j]);
        std::swap(x[pr], x[c]);
        det = -det;
      }
      det *= LU[(size_t)c * n + c];
      for (int q = c + 1; q < n; ++q) {
        const double fct = LU[(size_t)q * n + c] / LU[(size_t)c * n + c];
        for (int j = c; j < n; ++j) LU[(size_t)q * n + j] -= fct * LU[(size_t)c * n + j];
        x[q] -= fct * x[c];
      }
    }
    const long long vol = std::llround(std::fabs(det));
    if (vol == 0) return;
    for (int c = n - 1; c >= 0; --c) {
      double s = x[c];
      for (int j = c + 1; j < n; ++j) s -= LU[(size_t)c * n + j] * x[j];
      x[c] = s / LU[(size_t)c * n + c];
    }
    for (int k = 0; k < n; ++k) {
      const int i = order[k];
      const double base = w[i][ch[k].p];
      double hp = 0.0;
      for (int j = 0; j < n; ++j) hp += pts[i][ch[k].p][j] * x[j];
      for (size_t c = 0; c < pts[i].size(); ++c) {
        double hc = 0.0;
        for (int j = 0; j < n; ++j) hc += pts[i][c][j] * x[j];
        if (hc + w[i][c] < hp + base - 1e-9) return;
      }
    }
    mv += vol;
    if (cells != nullptr && ncells < max_cells)
      for (int k = 0; k < n; ++k) {
        cells[(size_t)ncells * 2 * n + 2 * order[k]] = ch[k].p;
        cells[(size_t)ncells * 2 * n + 2 * order[k] + 1] = ch[k].q;
      }
    ++ncells;
  }

  void extend(int level, std::vector<int> &sup, std::vector<Edge> &ch, std::vector<int> &idx) {
    const int i = order[level];
    for (int e = 0; e < (int)edges[i].size(); ++e) {
      bool ok = true;
      for (int k = 0; k < level && ok; ++k)
        ok = rel[(size_t)k * n + level][(size_t)idx[k] * edges[i].size() + e] != 0;
      if (!ok) continue;
      sup.push_back(i);
      ch.push_back(edges[i][e]);
      idx.push_back(e);
      if (level + 1 == n)
        leaf(ch);
      else if (level == 0 || feasible_choice(sup, ch))
        extend(level + 1, sup, ch, idx);
      sup.pop_back();
      ch.pop_back();
      idx.pop_back();
    }
  }
};

}  // namespace

extern "C" long long phc_mixed_volume(int n, const int *counts, const int *pts, unsigned long long seed,
                                      int max_cells, int *cells, long long *ncells) {
  PHC_REQUIRE(n >= 1 && n <= 64 && counts != nullptr && pts != nullptr, "mixed_volume: bad sizes");
  Search S;
  S.n = n;
  S.pts.resize(n);
  S.w.resize(n);
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 0x2545F4914F6CDD1Dull;
  auto rnd = [&]() {  // xorshift64*, uniform in [0, 1)
    st ^= st >> 12;
    st ^= st << 25;
    st ^= st >> 27;
    return (double)((st * 0x2545F4914F6CDD1Dull) >> 11) * (1.0 / 9007199254740992.0);
  };
  long off = 0;
  for (int i = 0; i < n; ++i) {
    PHC_REQUIRE(counts[i] >= 0 && counts[i] <= 100000, "mixed_volume: support %d has %d points", i, counts[i]);
    S.pts[i].assign(counts[i], std::vector<int>(n));
    for (int c = 0; c < counts[i]; ++c)
      for (int j = 0; j < n; ++j) S.pts[i][c][j] = pts[(off + c) * n + j];
    off += counts[i];
    S.w[i].resize(counts[i]);
    for (int c = 0; c < counts[i]; ++c) S.w[i][c] = rnd();
  }
  if (ncells) *ncells = 0;
  for (int i = 0; i < n; ++i)
    if (counts[i] < 2) return 0;
  // lower edges of each lifted support alone
  S.edges.resize(n);
  for (int i = 0; i < n; ++i)
    for (int p = 0; p < counts[i]; ++p)
      for (int q = p + 1; q < counts[i]; ++q) {
        std::vector<double> E, f, U, g;
        S.rows(i, Edge{p, q}, E, f, U, g);
        if (feasible(n, E, f, U, g)) S.edges[i].push_back(Edge{p, q});
      }
  S.order.resize(n);
  for (int i = 0; i < n; ++i) S.order[i] = i;
  std::stable_sort(S.order.begin(), S.order.end(),
                   [&](int a, int b) { return S.edges[a].size() < S.edges[b].size(); });
  // the relation table over the search order
  S.rel.assign((size_t)n * n, std::vector<char>());
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) {
      const int i = S.order[a], j = S.order[b];
      auto &t = S.rel[(size_t)a * n + b];
      t.assign(S.edges[i].size() * S.edges[j].size(), 0);
      for (size_t e = 0; e < S.edges[i].size(); ++e)
        for (size_t f = 0; f < S.edges[j].size(); ++f) {
          std::vector<double> E, fv, U, g;
          S.rows(i, S.edges[i][e], E, fv, U, g);
          S.rows(j, S.edges[j][f], E, fv, U, g);
          t[e * S.edges[j].size() + f] = feasible(n, E, fv, U, g) ? 1 : 0;
        }
    }
  S.max_cells = cells ? max_cells : 0;
  S.cells = cells;
  std::vector<int> sup, idx;
  std::vector<Edge> ch;
  S.extend(0, sup, ch, idx);
  if (ncells) *ncells = S.ncells;
  return S.mv;
}
