// manypaths.cu -- the tracker's drop-in entry points behind the phcpy / Ada
// C interface, gpumanypaths_d, gpumanypaths_dd and gpumanypaths_qd
// (Ada/PHCtoC/gpumanypaths_dd.h:27, body gpumanypaths_dd.cpp:18-62), and
// the containers they read and write.
//
// PHCpack's gpumanypaths_dd copies the target and the start system into its
// Ada system container, reads them and the start solutions out of the Ada
// containers (ada_read_sys, ada_read_sols), tracks every path of the
// artificial-parameter homotopy (1 - t) gamma q + t p and writes the end
// points back into the solution container (ada_write_sols).  The Ada
// containers need the Ada runtime; this library keeps containers of its own
// with the same content (the target system, the start system, the
// solutions), filled and read through phc_container_*, so that a caller
// (phcpy's py2c_gpu_manypaths_dd, or an adapter copying PHCpack's syscon /
// solcon contents) sets them, calls gpumanypaths_dd with the reference's
// arguments and reads the end points back.  Host code; the tracking is
// phc_track_host on the GPU.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include "common.cuh"
#include "tracker.cuh"
#include "../../include/phc_b200.h"

using namespace phc;

namespace {

struct PolyStore {
  int neq = 0, nvar = 0;
  std::vector<int> nterms, exps;  // terms per polynomial; nvar exponents per term
  std::vector<double> cff;        // complex double per term
  bool set = false;
};

struct SolStore {
  int nsols = 0, nvar = 0;
  std::vector<double> x;  // complex quad-double limbs: ((s*nvar + j)*2 + part)*4 + limb
  std::vector<double> t, res;
  std::vector<int> status;
  bool set = false;
};

std::mutex g_con_mu;
PolyStore g_target, g_start;
SolStore g_sols;
// tracking parameters (ipar, dpar of phc_track), defaults of the tracker
int g_ipar[7] = {8, 4, 4, 4, 3, 1000, 4};
double g_dpar[9] = {0.5, 1e-3, 0.1, 1e-6, 1e-8, 1e-12, 1e-24, 1.0, 0.005};

int store_poly(PolyStore &P, const char *who, int neq, int nvar, const int *nterms, const int *exps,
               const double *cff) {
  PHC_REQUIRE(neq >= 1 && nvar >= 1 && nterms != nullptr, "%s: need neq >= 1, nvar >= 1", who);
  long total = 0;
  for (int i = 0; i < neq; ++i) {
    PHC_REQUIRE(nterms[i] >= 0, "%s: polynomial %d has %d terms", who, i, nterms[i]);
    total += nterms[i];
  }
  PHC_REQUIRE(total == 0 || (exps != nullptr && cff != nullptr), "%s: null exponents or coefficients", who);
  for (long q = 0; q < total * nvar; ++q)
    PHC_REQUIRE(exps[q] >= 0, "%s: negative exponent in term %ld", who, q / nvar);
  P.neq = neq;
  P.nvar = nvar;
  P.nterms.assign(nterms, nterms + neq);
  P.exps.assign(exps, exps + total * nvar);
  P.cff.assign(cff, cff + 2 * total);
  P.set = true;
  return PHC_OK;
}

// The homotopy of phc_track for one target p and start system q (the
// arrays of include/phc_b200.h phc_track): the system's distinct monomials
// are the constant, then the target's and the start system's monomials in
// order of appearance; the terms of equation i follow that order, term r
// with a = gamma c_q, b = c_p.
struct Flat {
  int maxvar = 1;
  std::vector<int> dim, mono_off, nvr, idx, ex, eq_off, term_off, term_mono;
  std::vector<double> ta, tb;
};

int flatten(const PolyStore &p, const PolyStore &q, double gre, double gim, Flat &F) {
  const int n = p.nvar;
  typedef std::vector<int> Mono;  // exponent vector
  std::map<Mono, int> table;
  std::vector<Mono> order;
  auto id = [&](const Mono &m) {
    auto it = table.find(m);
    if (it != table.end()) return it->second;
    const int k = (int)order.size();
    table[m] = k;
    order.push_back(m);
    return k;
  };
  id(Mono(n, 0));
  for (const PolyStore *P : {&p, &q}) {
    long r = 0;
    for (int i = 0; i < P->neq; ++i)
      for (int k = 0; k < P->nterms[i]; ++k, ++r) id(Mono(P->exps.begin() + r * n, P->exps.begin() + (r + 1) * n));
  }
  int maxvar = 1;
  for (const Mono &m : order) {
    int c = 0;
    for (int e : m) c += e > 0;
    maxvar = c > maxvar ? c : maxvar;
  }
  F.maxvar = maxvar;
  F.dim = {n};
  F.mono_off = {0, (int)order.size()};
  for (const Mono &m : order) {
    int c = 0;
    for (int j = 0; j < n; ++j)
      if (m[j] > 0) {
        F.idx.push_back(j);
        F.ex.push_back(m[j]);
        ++c;
      }
    F.nvr.push_back(c);
    for (int v = c; v < maxvar; ++v) {
      F.idx.push_back(0);
      F.ex.push_back(0);
    }
  }
  // per equation: coefficients of the target and the start system per
  // monomial (repeated monomials add up), terms in monomial order
  long rp = 0, rq = 0;
  F.eq_off = {0, n};
  F.term_off = {0};
  for (int i = 0; i < n; ++i) {
    std::map<int, std::pair<double, double> > cp, cq;
    for (int k = 0; k < p.nterms[i]; ++k, ++rp) {
      auto &c = cp[table[Mono(p.exps.begin() + rp * n, p.exps.begin() + (rp + 1) * n)]];
      c.first += p.cff[2 * rp];
      c.second += p.cff[2 * rp + 1];
    }
    for (int k = 0; k < q.nterms[i]; ++k, ++rq) {
      auto &c = cq[table[Mono(q.exps.begin() + rq * n, q.exps.begin() + (rq + 1) * n)]];
      c.first += q.cff[2 * rq];
      c.second += q.cff[2 * rq + 1];
    }
    std::map<int, int> ids;
    for (auto &kv : cp) ids[kv.first] = 1;
    for (auto &kv : cq) ids[kv.first] = 1;
    for (auto &kv : ids) {
      const int m = kv.first;
      const std::pair<double, double> a0 = cq.count(m) ? cq[m] : std::make_pair(0.0, 0.0);
      const std::pair<double, double> b = cp.count(m) ? cp[m] : std::make_pair(0.0, 0.0);
      F.term_mono.push_back(m);
      F.ta.push_back(gre * a0.first - gim * a0.second);
      F.ta.push_back(gre * a0.second + gim * a0.first);
      F.tb.push_back(b.first);
      F.tb.push_back(b.second);
    }
    F.term_off.push_back((int)F.term_mono.size());
  }
  return PHC_OK;
}

// gpumanypaths_d, _dd and _qd: rmode is the refinement precision of the
// end points (2 for double and double-double, 4 for quad-double).
int manypaths(const char *who, int rmode, int mode, int verbose, double regamma, double imgamma) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  PHC_REQUIRE(mode == 0 || mode == 1 || mode == 2, "%s: mode %d not in {0, 1, 2}", who, mode);
  if (mode == 1) {
    set_error("%s: mode 1 runs the tracker on the CPU only; this library tracks on the GPU (modes 0 and 2)", who);
    return PHC_ERR_ARG;
  }
  PHC_REQUIRE(g_target.set && g_start.set && g_sols.set, "%s: the target system, the start system and the start "
              "solutions must be in the containers", who);
  const int n = g_target.nvar;
  PHC_REQUIRE(g_target.neq == n && g_start.neq == n && g_start.nvar == n && g_sols.nvar == n,
              "%s: need square systems of the same dimension as the solutions (%d equations, %d variables, start "
              "%d x %d, solutions of %d)", who, g_target.neq, n, g_start.neq, g_start.nvar, g_sols.nvar);
  PHC_REQUIRE(n <= 32, "%s: dimension %d above 32", who, n);
  const int npaths = g_sols.nsols;
  if (verbose > 0) {
    printf("\nAcceleration of tracking many paths ...\n");
    printf("gamma = %.16e + i* %.16e\n", regamma, imgamma);
    printf("Mode of execution : %d\n", mode);
    printf("number of polynomials : %d\n", n);
    printf("number of solutions : %d\n", npaths);
  }
  Flat F;
  int rc = flatten(g_target, g_start, regamma, imgamma, F);
  if (rc) return rc;
  std::vector<int> path_sys(npaths, 0);
  std::vector<double> x0((size_t)npaths * n * 2);
  for (int s = 0; s < npaths; ++s)
    for (int j = 0; j < n; ++j)
      for (int part = 0; part < 2; ++part) {
        const double *v = &g_sols.x[(((size_t)s * n + j) * 2 + part) * 4];
        x0[((size_t)s * n + j) * 2 + part] = v[0] + v[1];  // to the nearest double
      }
  std::vector<double> xend((size_t)npaths * n * 2 * 4), dinfo((size_t)npaths * 2);
  std::vector<int> info((size_t)npaths * kTrackInfo);
  if (npaths > 0) {
    rc = phc_track_host(1, F.dim.data(), F.maxvar, F.mono_off.data(), F.nvr.data(), F.idx.data(), F.ex.data(),
                        F.eq_off.data(), F.term_off.data(), F.term_mono.data(), F.ta.data(), F.tb.data(), npaths,
                        path_sys.data(), x0.data(), g_ipar, g_dpar, 1, rmode, 0, nullptr, xend.data(), info.data(),
                        dinfo.data(), nullptr);
    if (rc < 0) return rc;
  }
  if (verbose > 0) printf("writing the solutions to the container ...\n");
  g_sols.x = xend;
  g_sols.t.resize(npaths);
  g_sols.res.resize(npaths);
  g_sols.status.resize(npaths);
  for (int s = 0; s < npaths; ++s) {
    g_sols.status[s] = info[(size_t)kTrackInfo * s];
    g_sols.t[s] = dinfo[2 * s];
    g_sols.res[s] = dinfo[2 * s + 1];
  }
  return 0;
}

}  // namespace

extern "C" {

int phc_container_set_target(int neq, int nvar, const int *nterms, const int *exps, const double *cff) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  return store_poly(g_target, "container_set_target", neq, nvar, nterms, exps, cff);
}

int phc_container_set_start(int neq, int nvar, const int *nterms, const int *exps, const double *cff) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  return store_poly(g_start, "container_set_start", neq, nvar, nterms, exps, cff);
}

int phc_container_set_solutions(int nsols, int nvar, int limbs, const double *sols) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  PHC_REQUIRE(nsols >= 0 && nvar >= 1 && (limbs == 1 || limbs == 2 || limbs == 4),
              "container_set_solutions: need nsols >= 0, nvar >= 1, limbs in {1, 2, 4}");
  PHC_REQUIRE(nsols == 0 || sols != nullptr, "container_set_solutions: null solutions");
  g_sols.nsols = nsols;
  g_sols.nvar = nvar;
  g_sols.x.assign((size_t)nsols * nvar * 2 * 4, 0.0);
  for (long q = 0; q < (long)nsols * nvar * 2; ++q)
    for (int l = 0; l < limbs; ++l) g_sols.x[q * 4 + l] = sols[q * limbs + l];
  g_sols.t.assign(nsols, 0.0);
  g_sols.res.assign(nsols, 0.0);
  g_sols.status.assign(nsols, 0);
  g_sols.set = true;
  return PHC_OK;
}

int phc_container_number_of_solutions(int *nsols) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  PHC_REQUIRE(nsols != nullptr, "container_number_of_solutions: null pointer");
  *nsols = g_sols.set ? g_sols.nsols : 0;
  return PHC_OK;
}

int phc_container_dimension(int *nvar) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  PHC_REQUIRE(nvar != nullptr, "container_dimension: null pointer");
  *nvar = g_sols.set ? g_sols.nvar : (g_target.set ? g_target.nvar : 0);
  return PHC_OK;
}

int phc_container_get_solutions(int limbs, double *sols, double *t, int *status, double *res) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  PHC_REQUIRE(limbs == 1 || limbs == 2 || limbs == 4, "container_get_solutions: limbs %d not in {1, 2, 4}", limbs);
  PHC_REQUIRE(g_sols.set, "container_get_solutions: no solutions in the container");
  const long nq = (long)g_sols.nsols * g_sols.nvar * 2;
  if (sols)
    for (long q = 0; q < nq; ++q) {
      if (limbs == 1) {
        sols[q] = g_sols.x[q * 4] + g_sols.x[q * 4 + 1];
      } else {
        for (int l = 0; l < limbs; ++l) sols[q * limbs + l] = g_sols.x[q * 4 + l];
      }
    }
  for (int s = 0; s < g_sols.nsols; ++s) {
    if (t) t[s] = g_sols.t[s];
    if (status) status[s] = g_sols.status[s];
    if (res) res[s] = g_sols.res[s];
  }
  return PHC_OK;
}

int phc_container_set_parameters(const int *ipar, const double *dpar) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  PHC_REQUIRE(ipar != nullptr && dpar != nullptr, "container_set_parameters: null arrays");
  std::memcpy(g_ipar, ipar, sizeof(g_ipar));
  std::memcpy(g_dpar, dpar, sizeof(g_dpar));
  return PHC_OK;
}

void phc_container_clear(void) {
  std::lock_guard<std::mutex> lock(g_con_mu);
  g_target = PolyStore();
  g_start = PolyStore();
  g_sols = SolStore();
}

int gpumanypaths_d(int mode, int verbose, double regamma, double imgamma) {
  return manypaths("gpumanypaths_d", 2, mode, verbose, regamma, imgamma);
}

int gpumanypaths_dd(int mode, int verbose, double regamma, double imgamma) {
  return manypaths("gpumanypaths_dd", 2, mode, verbose, regamma, imgamma);
}

int gpumanypaths_qd(int mode, int verbose, double regamma, double imgamma) {
  return manypaths("gpumanypaths_qd", 4, mode, verbose, regamma, imgamma);
}

}  // extern "C"
