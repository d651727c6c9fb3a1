// capi_track.cu -- C ABI of the path tracker (include/phc_b200.h).
#include <cstring>
#include <mutex>
#include <vector>
#include "common.cuh"
#include "tracker.cuh"
#include "mlp.cuh"
#include "../../include/phc_b200.h"

namespace phc {
int track(const TrackDev &S, const TrackParDev &P, int nmono_max, int npaths, const int *path_sys, const double *x0,
          int pmode, int rmode, const void *model, double *xend, int *info, double *dinfo, float *log, int log_cap,
          int *log_count, int *queue, int one_per_launch, cudaStream_t st);
long track_smem_bytes(int maxdim, int K, int M, int nmono_max, int maxvar, int pmode, int rmode, int gst);
int track_check(const TrackParDev &P, int pmode, int rmode, int maxdim);
int series_diag(const TrackDev &S, const DiagParDev &D, int nmono_max, int npaths, const int *path_sys,
                const double *xpt, int xlimbs, const double *tpt, int pmode, double *series, double *dout, int *iout,
                cudaStream_t st);
int diag_check(const DiagParDev &D, int pmode, int maxdim, int xlimbs);
}  // namespace phc

using namespace phc;

namespace {
// The device buffer and the pinned staging buffer of phc_track_host, kept
// per device between calls and grown when a call needs more, so that a
// call of a size seen before allocates nothing; calls are serialised by the
// mutex (phc_track_host_release frees the buffers).
struct HostCallBuffers {
  void *dev = nullptr;
  size_t dev_cap = 0;
  void *pin = nullptr;
  size_t pin_cap = 0;
};
std::mutex g_track_mu;
HostCallBuffers g_track_buf[64];
}  // namespace

static TrackParDev make_par(const int *ipar, const double *dpar, int step_mode) {
  TrackParDev P;
  P.deg = ipar[0];
  P.numdeg = ipar[1];
  P.dendeg = ipar[2];
  P.nit = ipar[3];
  P.corsteps = ipar[4];
  P.maxsteps = ipar[5];
  P.refine_steps = ipar[6];
  P.step_mode = step_mode;
  P.pbeta = dpar[0];
  P.alpha = dpar[1];
  P.maxsize = dpar[2];
  P.minsize = dpar[3];
  P.tolres = dpar[4];
  P.epsilon = dpar[5];
  P.restol = dpar[6];
  P.learn_scale = dpar[7] > 0.0 ? dpar[7] : 1.0;
  P.cbeta = dpar[8];
  return P;
}

static DiagParDev make_diag_par(const int *ipar, const double *dpar) {
  DiagParDev D;
  D.deg = ipar[0];
  D.numdeg = ipar[1];
  D.dendeg = ipar[2];
  D.offset = ipar[3];
  D.newton_steps = ipar[4];
  D.tolres = dpar[0];
  D.beta2 = dpar[1];
  return D;
}

extern "C" {

long long phc_track_gather_count(int nsys, const int *mono_off, const int *mono_nvr, const int *eq_off,
                                 const int *term_off, const int *term_mono) {
  (void)mono_off;
  long long c = 0;
  const int neq = eq_off[nsys];
  for (int tr = 0; tr < term_off[neq]; ++tr) c += mono_nvr[term_mono[tr]];
  return c;
}

int phc_track_prepare(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr,
                      const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
                      const int *term_mono, int maxdim, int *jg_off, int *jg_term, int *jg_slot) {
  PHC_REQUIRE(nsys >= 0 && maxvar >= 1 && maxdim >= 1, "track_prepare: bad sizes");
  const int neq = eq_off[nsys];
  std::vector<std::vector<std::pair<int, int> > > lists((size_t)neq * maxdim);
  for (int s = 0; s < nsys; ++s) {
    PHC_REQUIRE(dim[s] >= 1 && dim[s] <= maxdim && eq_off[s + 1] - eq_off[s] == dim[s],
                "track_prepare: system %d has %d equations for dimension %d", s, eq_off[s + 1] - eq_off[s], dim[s]);
    for (int e = eq_off[s]; e < eq_off[s + 1]; ++e)
      for (int tr = term_off[e]; tr < term_off[e + 1]; ++tr) {
        const int m = term_mono[tr];
        PHC_REQUIRE(m >= mono_off[s] && m < mono_off[s + 1], "track_prepare: term %d uses monomial %d of another system", tr, m);
        PHC_REQUIRE(mono_nvr[m] >= 0 && mono_nvr[m] <= maxvar, "track_prepare: monomial %d has %d variables", m, mono_nvr[m]);
        for (int v = 0; v < mono_nvr[m]; ++v) {
          const int j = mono_idx[(long)m * maxvar + v];
          PHC_REQUIRE(j >= 0 && j < dim[s], "track_prepare: variable %d out of range in monomial %d", j, m);
          lists[(size_t)e * maxdim + j].push_back(std::make_pair(tr, v));
        }
      }
  }
  // slot codes: partials of monomials of total degree <= 2 are read in place
  int q = 0, staged = 0;
  for (size_t g = 0; g < lists.size(); ++g) {
    jg_off[g] = q;
    for (auto &pr : lists[g]) {
      const int m = term_mono[pr.first], v = pr.second;
      const int *ix = mono_idx + (long)m * maxvar, *ex = mono_exp + (long)m * maxvar;
      int code = v;
      if (simple_monomial(mono_nvr[m], ex))
        code = mono_nvr[m] == 1 ? (ex[0] == 1 ? -1 : -2) : -3 - ix[1 - v];
      else
        ++staged;
      jg_term[q] = pr.first;
      jg_slot[q] = code;
      ++q;
    }
  }
  jg_off[lists.size()] = q;
  return staged;
}

long long phc_track_smem_bytes(int maxdim, int deg, int dendeg, int nmono_max, int maxvar, int pmode, int rmode, int gstaged) {
  return track_smem_bytes(maxdim, deg, dendeg, nmono_max, maxvar, pmode, rmode, gstaged);
}

long long phc_mlp_model_bytes(void) { return mlp_model_bytes(); }

int phc_track(int nsys, const int *dim, int maxvar, int maxdim, int nmono_max, const int *mono_off,
              const int *mono_nvr, const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
              const int *term_mono, const double *term_a, const double *term_b, const int *jg_off,
              const int *jg_term, const int *jg_slot, int gstaged, int npaths, const int *path_sys,
              const double *x0, const int *ipar, const double *dpar, int pmode, int rmode, int step_mode,
              const void *model, double *xend, int *info, double *dinfo, float *log, int log_cap, int *log_count,
              int *queue, int one_per_launch, void *stream) {
  TrackDev S{nsys,      maxvar, maxdim, dim,    mono_off, mono_nvr, mono_idx, mono_exp,    eq_off,
             term_off,  term_mono, term_a, term_b, jg_off,  jg_term,  jg_slot,  gstaged != 0};
  return track(S, make_par(ipar, dpar, step_mode), nmono_max, npaths, path_sys, x0, pmode, rmode,
               (step_mode & 1) ? model : nullptr, xend, info, dinfo, log, log_cap, log_count, queue, one_per_launch,
               (cudaStream_t)stream);
}

int phc_track_host(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr,
                   const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
                   const int *term_mono, const double *term_a, const double *term_b, int npaths,
                   const int *path_sys, const double *x0, const int *ipar, const double *dpar, int pmode, int rmode,
                   int step_mode, const void *model, double *xend, int *info, double *dinfo, void *stream) {
  PHC_REQUIRE(nsys >= 1 && npaths >= 0, "track_host: bad sizes");
  int maxdim = 0, nmono_max = 0;
  for (int s = 0; s < nsys; ++s) {
    maxdim = dim[s] > maxdim ? dim[s] : maxdim;
    nmono_max = (mono_off[s + 1] - mono_off[s]) > nmono_max ? (mono_off[s + 1] - mono_off[s]) : nmono_max;
  }
  // the checks of phc_track, made here before any device work
  {
    const TrackParDev P = make_par(ipar, dpar, step_mode);
    const int rc = track_check(P, pmode, rmode, maxdim);
    if (rc) return rc;
  }
  const int neq = eq_off[nsys];
  const int nterm = term_off[neq];
  const int nmono = mono_off[nsys];
  const long long njg = phc_track_gather_count(nsys, mono_off, mono_nvr, eq_off, term_off, term_mono);
  std::vector<int> jg_off((size_t)neq * maxdim + 1), jg_term(njg > 0 ? njg : 1), jg_slot(njg > 0 ? njg : 1);
  const int staged = phc_track_prepare(nsys, dim, maxvar, mono_off, mono_nvr, mono_idx, mono_exp, eq_off, term_off,
                                       term_mono, maxdim, jg_off.data(), jg_term.data(), jg_slot.data());
  if (staged < 0) return staged;
  // one device buffer for everything, staged through one pinned host buffer
  std::vector<std::pair<const void *, size_t> > ins = {
      {dim, nsys * 4ul}, {mono_off, (nsys + 1) * 4ul}, {mono_nvr, nmono * 4ul},
      {mono_idx, (size_t)nmono * maxvar * 4}, {mono_exp, (size_t)nmono * maxvar * 4}, {eq_off, (nsys + 1) * 4ul},
      {term_off, (neq + 1) * 4ul}, {term_mono, nterm * 4ul}, {term_a, nterm * 16ul}, {term_b, nterm * 16ul},
      {jg_off.data(), jg_off.size() * 4}, {jg_term.data(), jg_term.size() * 4}, {jg_slot.data(), jg_slot.size() * 4},
      {path_sys, npaths * 4ul}, {x0, (size_t)npaths * maxdim * 16},
      {model, (step_mode & 1) && model ? (size_t)mlp_model_bytes() : 0ul}};
  size_t total = 0;
  std::vector<size_t> off;
  for (size_t i = 0; i < ins.size(); ++i) {
    off.push_back(total);
    total += (ins[i].second + 255) & ~size_t(255);
  }
  const size_t xbytes = (size_t)npaths * maxdim * (rmode == 8 ? 128 : 64);  // complex qd (od) per coordinate
  const size_t o_xend = total;
  total += (xbytes + 255) & ~size_t(255);
  const size_t o_info = total;
  total += (((size_t)npaths * 4 * kTrackInfo) + 255) & ~size_t(255);
  const size_t o_dinfo = total;
  total += (((size_t)npaths * 16) + 255) & ~size_t(255);
  const size_t o_q = total;
  total += 256;
  const size_t in_bytes = o_xend, out_bytes = o_q - o_xend;
  int devid = 0;
  PHC_CUDA(cudaGetDevice(&devid));
  if (devid < 0 || devid >= 64) {
    set_error("track_host: device %d beyond the 64 whose buffers are kept", devid);
    return PHC_ERR_LIMIT;
  }
  std::lock_guard<std::mutex> lock(g_track_mu);
  HostCallBuffers &hb = g_track_buf[devid];
  if (hb.dev_cap < total) {
    if (hb.dev) cudaFree(hb.dev);
    hb.dev = nullptr;
    hb.dev_cap = 0;
    PHC_CUDA(cudaMalloc(&hb.dev, total));
    hb.dev_cap = total;
  }
  const size_t pin_need = in_bytes > out_bytes ? in_bytes : out_bytes;
  if (hb.pin_cap < pin_need) {
    if (hb.pin) cudaFreeHost(hb.pin);
    hb.pin = nullptr;
    hb.pin_cap = 0;
    PHC_CUDA(cudaMallocHost(&hb.pin, pin_need));
    hb.pin_cap = pin_need;
  }
  char *b = (char *)hb.dev, *h = (char *)hb.pin;
  for (size_t i = 0; i < ins.size(); ++i)
    if (ins[i].second) std::memcpy(h + off[i], ins[i].first, ins[i].second);
  cudaStream_t st = (cudaStream_t)stream;
  int out = PHC_OK;
  if (cudaMemcpyAsync(b, h, in_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
    set_error("track_host: copy to the device failed");
    out = PHC_ERR_CUDA;
  }
  if (out == PHC_OK) {
    auto I = [&](int i) { return (const int *)(b + off[i]); };
    auto Dp = [&](int i) { return (const double *)(b + off[i]); };
    out = phc_track(nsys, I(0), maxvar, maxdim, nmono_max, I(1), I(2), I(3), I(4), I(5), I(6), I(7), Dp(8), Dp(9),
                    I(10), I(11), I(12), staged, npaths, I(13), Dp(14), ipar, dpar, pmode, rmode, step_mode,
                    (step_mode & 1) && model ? (const void *)(b + off[15]) : nullptr, (double *)(b + o_xend),
                    (int *)(b + o_info), (double *)(b + o_dinfo), nullptr, 0, nullptr, (int *)(b + o_q), 0, st);
  }
  if (out == PHC_OK) {
    if (cudaMemcpyAsync(h, b + o_xend, out_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      set_error("track_host: %s", cudaGetErrorString(cudaGetLastError()));
      out = PHC_ERR_CUDA;
    } else {
      std::memcpy(xend, h, xbytes);
      std::memcpy(info, h + (o_info - o_xend), (size_t)npaths * 4 * kTrackInfo);
      std::memcpy(dinfo, h + (o_dinfo - o_xend), (size_t)npaths * 16);
    }
  }
  if (out < 0) return out;
  int fails = 0;
  for (int p = 0; p < npaths; ++p) fails += info[(long)kTrackInfo * p] != 0;
  return fails;
}

void phc_track_host_release(void) {
  std::lock_guard<std::mutex> lock(g_track_mu);
  int cur = 0;
  cudaGetDevice(&cur);
  for (int d = 0; d < 64; ++d) {
    HostCallBuffers &hb = g_track_buf[d];
    if (!hb.dev && !hb.pin) continue;
    cudaSetDevice(d);
    if (hb.dev) cudaFree(hb.dev);
    if (hb.pin) cudaFreeHost(hb.pin);
    hb = HostCallBuffers();
  }
  cudaSetDevice(cur);
}

int phc_series_diagnostics(int nsys, const int *dim, int maxvar, int maxdim, int nmono_max, const int *mono_off,
                           const int *mono_nvr, const int *mono_idx, const int *mono_exp, const int *eq_off,
                           const int *term_off, const int *term_mono, const double *term_a, const double *term_b,
                           const int *jg_off, const int *jg_term, const int *jg_slot, int gstaged, int npaths,
                           const int *path_sys, const double *xpt, int xlimbs, const double *tpt, const int *ipar,
                           const double *dpar, int pmode, double *series, double *dout, int *iout, void *stream) {
  PHC_REQUIRE(nsys >= 1 && npaths >= 0, "series_diagnostics: bad sizes");
  TrackDev S{nsys,      maxvar, maxdim, dim,    mono_off, mono_nvr, mono_idx, mono_exp,    eq_off,
             term_off,  term_mono, term_a, term_b, jg_off,  jg_term,  jg_slot,  gstaged != 0};
  return series_diag(S, make_diag_par(ipar, dpar), nmono_max, npaths, path_sys, xpt, xlimbs, tpt, pmode, series,
                     dout, iout, (cudaStream_t)stream);
}

int phc_series_diagnostics_host(int nsys, const int *dim, int maxvar, const int *mono_off, const int *mono_nvr,
                                const int *mono_idx, const int *mono_exp, const int *eq_off, const int *term_off,
                                const int *term_mono, const double *term_a, const double *term_b, int npaths,
                                const int *path_sys, const double *xpt, int xlimbs, const double *tpt,
                                const int *ipar, const double *dpar, int pmode, double *series, double *dout,
                                int *iout) {
  PHC_REQUIRE(nsys >= 1 && npaths >= 0, "series_diagnostics_host: bad sizes");
  int maxdim = 0, nmono_max = 0;
  for (int s = 0; s < nsys; ++s) {
    maxdim = dim[s] > maxdim ? dim[s] : maxdim;
    nmono_max = (mono_off[s + 1] - mono_off[s]) > nmono_max ? (mono_off[s + 1] - mono_off[s]) : nmono_max;
  }
  const DiagParDev D = make_diag_par(ipar, dpar);
  {
    const int rc = diag_check(D, pmode, maxdim, xlimbs);
    if (rc) return rc;
  }
  if (npaths == 0) return PHC_OK;
  const int neq = eq_off[nsys];
  const int nterm = term_off[neq];
  const int nmono = mono_off[nsys];
  const long long njg = phc_track_gather_count(nsys, mono_off, mono_nvr, eq_off, term_off, term_mono);
  std::vector<int> jg_off((size_t)neq * maxdim + 1), jg_term(njg > 0 ? njg : 1), jg_slot(njg > 0 ? njg : 1);
  const int staged = phc_track_prepare(nsys, dim, maxvar, mono_off, mono_nvr, mono_idx, mono_exp, eq_off, term_off,
                                       term_mono, maxdim, jg_off.data(), jg_term.data(), jg_slot.data());
  if (staged < 0) return staged;
  const size_t sbytes = (size_t)npaths * maxdim * (D.deg + 1) * 2 * pmode * sizeof(double);
  std::vector<std::pair<const void *, size_t> > ins = {
      {dim, nsys * 4ul}, {mono_off, (nsys + 1) * 4ul}, {mono_nvr, nmono * 4ul},
      {mono_idx, (size_t)nmono * maxvar * 4}, {mono_exp, (size_t)nmono * maxvar * 4}, {eq_off, (nsys + 1) * 4ul},
      {term_off, (neq + 1) * 4ul}, {term_mono, nterm * 4ul}, {term_a, nterm * 16ul}, {term_b, nterm * 16ul},
      {jg_off.data(), jg_off.size() * 4}, {jg_term.data(), jg_term.size() * 4}, {jg_slot.data(), jg_slot.size() * 4},
      {path_sys, npaths * 4ul}, {xpt, (size_t)npaths * maxdim * 2 * xlimbs * 8}, {tpt, npaths * 8ul}};
  std::vector<size_t> off;
  size_t total = 0;
  for (auto &in : ins) {
    off.push_back(total);
    total += (in.second + 255) & ~size_t(255);
  }
  const size_t o_series = total;
  total += (sbytes + 255) & ~size_t(255);
  const size_t o_dout = total;
  total += ((size_t)npaths * kDiagOut * 8 + 255) & ~size_t(255);
  const size_t o_iout = total;
  total += ((size_t)npaths * 8 + 255) & ~size_t(255);
  char *b = nullptr;
  PHC_CUDA(cudaMalloc((void **)&b, total));
  int out = PHC_OK;
  for (size_t i = 0; i < ins.size() && out == PHC_OK; ++i)
    if (ins[i].second && cudaMemcpy(b + off[i], ins[i].first, ins[i].second, cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("series_diagnostics_host: copy to the device failed");
      out = PHC_ERR_CUDA;
    }
  if (out == PHC_OK && series && cudaMemset(b + o_series, 0, sbytes) != cudaSuccess) {
    set_error("series_diagnostics_host: memset failed");
    out = PHC_ERR_CUDA;
  }
  if (out == PHC_OK) {
    auto I = [&](int i) { return (const int *)(b + off[i]); };
    auto Dp = [&](int i) { return (const double *)(b + off[i]); };
    out = phc_series_diagnostics(nsys, I(0), maxvar, maxdim, nmono_max, I(1), I(2), I(3), I(4), I(5), I(6), I(7),
                                 Dp(8), Dp(9), I(10), I(11), I(12), staged, npaths, I(13), Dp(14), xlimbs, Dp(15),
                                 ipar, dpar, pmode, series ? (double *)(b + o_series) : nullptr,
                                 (double *)(b + o_dout), (int *)(b + o_iout), nullptr);
  }
  if (out == PHC_OK) {
    if (cudaMemcpy(dout, b + o_dout, (size_t)npaths * kDiagOut * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(iout, b + o_iout, (size_t)npaths * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        (series && cudaMemcpy(series, b + o_series, sbytes, cudaMemcpyDeviceToHost) != cudaSuccess)) {
      set_error("series_diagnostics_host: %s", cudaGetErrorString(cudaGetLastError()));
      out = PHC_ERR_CUDA;
    }
  }
  cudaFree(b);
  return out;
}

}  // extern "C"
