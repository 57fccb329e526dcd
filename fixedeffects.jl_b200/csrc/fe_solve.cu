// fe_solve.cu -- tile dispatch of the solve drivers (fe_solve_impl.cuh) and
// the per-column verdicts of a solve.
#include <cuda_runtime.h>

#include <sys/stat.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "fe_plan.h"
#include "fe_solve.h"

namespace fe {

template <int C>
int solve_tile_C(fe_plan* pl, const SolveReq& rq, int64_t col0, int ncols, std::vector<Inst>& out);
extern template int solve_tile_C<1>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
extern template int solve_tile_C<2>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
extern template int solve_tile_C<4>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
extern template int solve_tile_C<8>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
extern template int solve_tile_C<16>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
extern template int solve_tile_C<32>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
int prof_flush(fe_plan* pl) {
  if (pl->prof.pending.empty()) return 0;
  FE_CK(cudaStreamSynchronize(pl->stream));
  for (auto& pr : pl->prof.pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pr.second.first, pr.second.second);
    KernelStat& st = pl->prof.stats[pr.first];
    st.name = pr.first;
    st.launches += 1;
    st.ms += ms;
    st.times.push_back(ms);
    st.bytes += pl->prof.bytes_per_launch[pr.first];
    pl->prof.pool.push_back(pr.second.first);
    pl->prof.pool.push_back(pr.second.second);
  }
  pl->prof.pending.clear();
  return 0;
}

// ---------------------------------------------------------------------------
// persisted tuning cache: one line per tuned tile shape,
//   <signature> <C> <element size> <expand variant> <segsum variant>
// in $FE_B200_TUNE_CACHE (a path; "off" disables), else
// $XDG_CACHE_HOME/fe_b200/tune.txt or $HOME/.cache/fe_b200/tune.txt.
// ---------------------------------------------------------------------------
static std::string tune_cache_path() {
  const char* e = std::getenv("FE_B200_TUNE_CACHE");
  if (e && *e) {
    const std::string v(e);
    if (v == "off" || v == "0") return std::string();
    return v;
  }
  std::string dir;
  if (const char* x = std::getenv("XDG_CACHE_HOME")) dir = x;
  else if (const char* h = std::getenv("HOME")) dir = std::string(h) + "/.cache";
  else return std::string();
  return dir + "/fe_b200/tune.txt";
}

static const std::string& tune_signature(fe_plan* pl) {
  if (pl->tune_signature.empty()) {
    cudaDeviceProp prop;
    std::ostringstream os;
    if (cudaGetDeviceProperties(&prop, pl->device) == cudaSuccess) {
      std::string name(prop.name);
      for (char& ch : name)
        if (ch == ' ') ch = '_';
      os << name << "/sm" << prop.multiProcessorCount;
    } else {
      (void)cudaGetLastError();
      os << "unknown";
    }
    os << "/kv3/N" << pl->N << "/P" << pl->nprob << "/K" << pl->K << "/w" << (pl->weighted ? 1 : 0);
    for (int k = 0; k < pl->K; ++k) os << "/" << pl->nlev[k] << (pl->interacted[k] ? "i" : "");
    pl->tune_signature = os.str();
  }
  return pl->tune_signature;
}

bool tune_cache_load(fe_plan* pl, int C, int sT, int* ex, int* seg) {
  const std::string path = tune_cache_path();
  if (path.empty()) return false;
  std::ifstream f(path);
  if (!f) return false;
  const std::string& sig = tune_signature(pl);
  std::string line;
  bool found = false;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string s;
    int c = 0, t = 0, e = 0, g = 0;
    if (!(is >> s >> c >> t >> e >> g)) continue;
    if (s == sig && c == C && t == sT && e >= 0 && e < 6 && g >= 0 && g < 6) {
      *ex = e;
      *seg = g;
      found = true;  // the last matching line wins
    }
  }
  return found;
}

void tune_cache_store(fe_plan* pl, int C, int sT, int ex, int seg) {
  const std::string path = tune_cache_path();
  if (path.empty()) return;
  // create the parent directories (best effort)
  for (size_t pos = path.find('/', 1); pos != std::string::npos; pos = path.find('/', pos + 1))
    mkdir(path.substr(0, pos).c_str(), 0755);
  std::ofstream f(path, std::ios::app);
  if (f) f << tune_signature(pl) << " " << C << " " << sT << " " << ex << " " << seg << "\n";
}

int tile_width(const fe_plan* pl, int64_t remaining) {
  int cmax = 32;
  if (pl->opt_tile > 0) cmax = pl->opt_tile;
  int64_t want = std::min<int64_t>(remaining, cmax);
  int C = 1;
  while (C < want) C <<= 1;
  return std::min(C, 32);
}

int solve(fe_plan* pl, const SolveReq& rq) {
  NvtxRange nv(rq.residuals ? "fe: solve_residuals" : "fe: solve_coefficients");
  FE_CK(cudaSetDevice(pl->device));
  const int64_t ncols = rq.ncols;
  pl->last_test2.assign((size_t)ncols, 0.0);
  pl->last_rounds.assign((size_t)ncols, 0);
  pl->last_iters_raw.assign((size_t)ncols, 0);
  if (pl->N == 0) {
    for (int64_t j = 0; j < ncols; ++j) {
      if (rq.iters) rq.iters[j] = rq.residuals ? 1 : 0;
      if (rq.converged) rq.converged[j] = 1;
    }
    return 0;
  }
  std::vector<Inst> res;
  for (int64_t col0 = 0; col0 < ncols;) {
    const int C = tile_width(pl, ncols - col0);
    const int nc = (int)std::min<int64_t>(C, ncols - col0);
    int st;
    if (rq.before_tile && (st = rq.before_tile(rq.hook_ctx, col0, nc))) return st;
    switch (C) {
      case 1: st = solve_tile_C<1>(pl, rq, col0, nc, res); break;
      case 2: st = solve_tile_C<2>(pl, rq, col0, nc, res); break;
      case 4: st = solve_tile_C<4>(pl, rq, col0, nc, res); break;
      case 8: st = solve_tile_C<8>(pl, rq, col0, nc, res); break;
      case 16: st = solve_tile_C<16>(pl, rq, col0, nc, res); break;
      default: st = solve_tile_C<32>(pl, rq, col0, nc, res); break;
    }
    if (st) return st;
    if (rq.after_tile && (st = rq.after_tile(rq.hook_ctx, col0, nc))) return st;
    // per-column verdicts: a column's instances are (problem p, column j);
    // with several problems the column aggregates them (max iterations, all
    // converged).  Single-problem plans report the instance itself.
    for (int j = 0; j < nc; ++j) {
      int64_t itmax = 0, raw = 0;
      bool conv = true;
      double t2 = 0.0;
      int32_t rounds = 0;
      for (int p = 0; p < pl->nprob; ++p) {
        const Inst& s = res[(size_t)p * C + j];
        int64_t it;
        bool cv;
        if (rq.precision == 1) {
          raw = std::max<int64_t>(raw, s.iter_total);
          it = rq.residuals ? s.iter_total + 1 : s.iter_total / 2;
          cv = s.converged != 0;
          t2 = std::max(t2, s.last_test2);
          rounds = std::max(rounds, s.outer_rounds);
        } else {
          raw = std::max<int64_t>(raw, s.iter);
          it = rq.residuals ? (s.skip_lsmr ? 1 : s.iter + 1) : s.iter / 2;
          cv = !(s.istop == 3 || s.istop == 6 || s.istop == 7);
        }
        itmax = std::max(itmax, it);
        conv = conv && cv;
        if (rq.prob_iters) rq.prob_iters[(size_t)p * ncols + col0 + j] = it;
        if (rq.prob_converged) rq.prob_converged[(size_t)p * ncols + col0 + j] = cv ? 1 : 0;
      }
      if (rq.iters) rq.iters[col0 + j] = itmax;
      if (rq.converged) rq.converged[col0 + j] = conv ? 1 : 0;
      pl->last_test2[(size_t)(col0 + j)] = t2;
      pl->last_rounds[(size_t)(col0 + j)] = rounds;
      pl->last_iters_raw[(size_t)(col0 + j)] = raw;
    }
    col0 += nc;
  }
  return 0;
}

}  // namespace fe
