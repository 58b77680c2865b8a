// mtp_model.cpp - .mtp parsing and contraction-schedule construction (host).
#include "mtp_model.hpp"

#include <algorithm>
#include <array>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <numeric>
#include <queue>
#include <sstream>

namespace mtp {

// ---------------------------------------------------------------------------
// .mtp parsing (format of motep_original_files/mtp.py:31-70)
// ---------------------------------------------------------------------------
namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

bool parse_int(const std::string& s, int& v) {
  std::string t = trim(s);
  if (t.empty()) return false;
  char* end = nullptr;
  long x = std::strtol(t.c_str(), &end, 10);
  if (*end != '\0' || x < INT_MIN || x > INT_MAX) return false;
  v = static_cast<int>(x);
  return true;
}

bool parse_double(const std::string& s, double& v) {
  std::string t = trim(s);
  if (t.empty()) return false;
  char* end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return *end == '\0';
}

// "{a, b, c}" -> numbers
template <typename T>
bool parse_list(const std::string& s, std::vector<T>& out) {
  std::string t = trim(s);
  if (t.size() < 2 || t.front() != '{' || t.back() != '}') return false;
  out.clear();
  const char* p = t.c_str() + 1;
  const char* e = t.c_str() + t.size() - 1;
  while (p < e) {
    while (p < e && (std::isspace(static_cast<unsigned char>(*p)) || *p == ',')) ++p;
    if (p >= e) break;
    char* end = nullptr;
    double x = std::strtod(p, &end);
    if (end == p) return false;
    out.push_back(static_cast<T>(x));
    if (std::is_integral<T>::value && x != std::floor(x)) return false;
    p = end;
  }
  return true;
}

// "{{a,b,c,d}, {...}}" -> flat ints, 4 per row
bool parse_table(const std::string& s, std::vector<int>& out) {
  std::string t = trim(s);
  if (t.size() < 2 || t.front() != '{' || t.back() != '}') return false;
  out.clear();
  const char* p = t.c_str() + 1;
  const char* e = t.c_str() + t.size() - 1;
  while (p < e) {
    while (p < e && *p != '{') {
      if (!std::isspace(static_cast<unsigned char>(*p)) && *p != ',') return false;
      ++p;
    }
    if (p >= e) break;
    ++p;  // '{'
    int n = 0;
    while (p < e && *p != '}') {
      while (p < e && (std::isspace(static_cast<unsigned char>(*p)) || *p == ',')) ++p;
      if (*p == '}') break;
      char* end = nullptr;
      long x = std::strtol(p, &end, 10);
      if (end == p) return false;
      out.push_back(static_cast<int>(x));
      ++n;
      p = end;
    }
    if (p >= e || *p != '}' || n != 4) return false;
    ++p;
  }
  return true;
}

}  // namespace

bool parse_mtp_text(const std::string& text, Potential& pot, std::string& err) {
  pot = Potential();
  std::vector<std::string> lines;
  {
    std::istringstream is(text);
    std::string l;
    while (std::getline(is, l)) lines.push_back(l);
  }
  bool header = false, have_radial = false;
  bool have_basic = false, have_times = false, have_map = false, have_sp = false, have_mc = false;
  int basic_count = -1, times_count = -1;
  for (size_t i = 0; i < lines.size(); ++i) {
    std::string line = trim(lines[i]);
    if (line.empty()) continue;
    if (line == "MTP") { header = true; continue; }
    if (line == "radial_coeffs") {
      if (pot.S <= 0 || pot.R <= 0 || pot.K <= 0) {
        err = "radial_coeffs block before species_count/radial_funcs_count/radial_basis_size";
        return false;
      }
      pot.radial.assign(static_cast<size_t>(pot.S) * pot.S * pot.R * pot.K, NAN);
      std::vector<char> seen(static_cast<size_t>(pot.S) * pot.S, 0);
      for (int pair = 0; pair < pot.S * pot.S; ++pair) {
        if (++i >= lines.size()) { err = "truncated radial_coeffs block"; return false; }
        std::string hdr = trim(lines[i]);
        size_t dash = hdr.find('-');
        int a = -1, b = -1;
        if (dash == std::string::npos || !parse_int(hdr.substr(0, dash), a) ||
            !parse_int(hdr.substr(dash + 1), b) || a < 0 || b < 0 || a >= pot.S || b >= pot.S) {
          err = "bad species pair line '" + hdr + "' in radial_coeffs";
          return false;
        }
        seen[a * pot.S + b] = 1;
        for (int mu = 0; mu < pot.R; ++mu) {
          if (++i >= lines.size()) { err = "truncated radial_coeffs block"; return false; }
          std::vector<double> row;
          if (!parse_list(lines[i], row) || static_cast<int>(row.size()) != pot.K) {
            err = "radial_coeffs row must hold radial_basis_size numbers";
            return false;
          }
          std::copy(row.begin(), row.end(),
                    pot.radial.begin() + ((static_cast<size_t>(a) * pot.S + b) * pot.R + mu) * pot.K);
        }
      }
      for (char c : seen)
        if (!c) { err = "radial_coeffs does not cover every species pair"; return false; }
      have_radial = true;
      continue;
    }
    size_t eq = line.find('=');
    if (eq == std::string::npos) { err = "unrecognised line '" + line.substr(0, 60) + "'"; return false; }
    std::string key = trim(line.substr(0, eq));
    std::string val = trim(line.substr(eq + 1));
    bool ok = true;
    if (key == "version") pot.version = val;
    else if (key == "potential_name") pot.potential_name = val;
    else if (key == "potential_tag") pot.potential_tag = val;
    else if (key == "radial_basis_type") pot.radial_basis_type = val;
    else if (key == "scaling") ok = parse_double(val, pot.scaling);
    else if (key == "min_dist") ok = parse_double(val, pot.min_dist);
    else if (key == "max_dist") ok = parse_double(val, pot.max_dist);
    else if (key == "species_count") ok = parse_int(val, pot.S);
    else if (key == "radial_basis_size") ok = parse_int(val, pot.K);
    else if (key == "radial_funcs_count") ok = parse_int(val, pot.R);
    else if (key == "alpha_moments_count") ok = parse_int(val, pot.M);
    else if (key == "alpha_index_basic_count") ok = parse_int(val, basic_count);
    else if (key == "alpha_index_times_count") ok = parse_int(val, times_count);
    else if (key == "alpha_scalar_moments") ok = parse_int(val, pot.Sa);
    else if (key == "alpha_index_basic") { ok = parse_table(val, pot.basic); have_basic = ok; }
    else if (key == "alpha_index_times") { ok = parse_table(val, pot.times); have_times = ok; }
    else if (key == "alpha_moment_mapping") { ok = parse_list(val, pot.mapping); have_map = ok; }
    else if (key == "species_coeffs") { ok = parse_list(val, pot.species); have_sp = ok; }
    else if (key == "moment_coeffs") { ok = parse_list(val, pot.moment); have_mc = ok; }
    // unknown keys are ignored, as the reference stores them as strings
    if (!ok) { err = "bad value for '" + key + "'"; return false; }
  }
  if (!header) { err = "missing 'MTP' header line"; return false; }
  if (pot.radial_basis_type != "RBChebyshev") {
    err = "radial_basis_type '" + pot.radial_basis_type + "' is not RBChebyshev";
    return false;
  }
  if (!have_radial) { err = "missing radial_coeffs (an untrained template has no coefficients)"; return false; }
  if (!have_basic || !have_times || !have_map || !have_sp || !have_mc) {
    err = "missing one of alpha_index_basic, alpha_index_times, alpha_moment_mapping, species_coeffs, moment_coeffs";
    return false;
  }
  pot.B = static_cast<int>(pot.basic.size() / 4);
  pot.T = static_cast<int>(pot.times.size() / 4);
  if (basic_count >= 0 && basic_count != pot.B) { err = "alpha_index_basic_count does not match the table"; return false; }
  if (times_count >= 0 && times_count != pot.T) { err = "alpha_index_times_count does not match the table"; return false; }
  if (static_cast<int>(pot.mapping.size()) != pot.Sa) { err = "alpha_scalar_moments does not match alpha_moment_mapping"; return false; }
  if (static_cast<int>(pot.moment.size()) != pot.Sa) { err = "moment_coeffs must have alpha_scalar_moments entries"; return false; }
  if (static_cast<int>(pot.species.size()) != pot.S) { err = "species_coeffs must have species_count entries"; return false; }
  if (pot.S <= 0 || pot.R <= 0 || pot.K <= 0 || pot.M <= 0) { err = "non-positive basis sizes"; return false; }
  if (pot.R > kMaxR) { err = "radial_funcs_count above the supported 8"; return false; }
  if (pot.K > kMaxK) { err = "radial_basis_size above the supported 16"; return false; }
  if (!(pot.max_dist > pot.min_dist) || !(pot.max_dist > 0.0)) { err = "need max_dist > min_dist and max_dist > 0"; return false; }
  if (pot.B > pot.M) { err = "more basic moments than moments"; return false; }
  for (int k = 0; k < pot.B; ++k) {
    const int* r = &pot.basic[4 * k];
    if (r[0] < 0 || r[0] >= pot.R || r[1] < 0 || r[2] < 0 || r[3] < 0) {
      err = "alpha_index_basic row out of range"; return false;
    }
    if (r[1] + r[2] + r[3] > kMaxDegree) { err = "monomial degree above the supported 12"; return false; }
  }
  for (int e = 0; e < pot.T; ++e) {
    const int* r = &pot.times[4 * e];
    if (r[0] < 0 || r[0] >= pot.M || r[1] < 0 || r[1] >= pot.M || r[3] < 0 || r[3] >= pot.M) {
      err = "alpha_index_times refers to a moment out of range"; return false;
    }
  }
  for (int v : pot.mapping)
    if (v < 0 || v >= pot.M) { err = "alpha_moment_mapping refers to a moment out of range"; return false; }
  for (double v : pot.radial)
    if (!std::isfinite(v)) { err = "non-finite radial coefficient"; return false; }
  return true;
}

bool parse_mtp_file(const std::string& path, Potential& pot, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) { err = "cannot open '" + path + "'"; return false; }
  std::stringstream ss;
  ss << f.rdbuf();
  return parse_mtp_text(ss.str(), pot, err);
}

// ---------------------------------------------------------------------------
// schedule
// ---------------------------------------------------------------------------
namespace {

// Symbolic value-space operands resolved after the partial count is known.
constexpr uint32_t kSymZero = 0x80000000u;
constexpr uint32_t kSymOne = 0x80000001u;
constexpr uint32_t kSymPartBase = 0xC0000000u;

struct Side {
  uint32_t a, b;
  uint32_t c;
};
struct Job {
  uint32_t dst;
  uint32_t op;
  std::vector<Side> sides;
};
struct RawEntry {
  uint32_t a, b, dst, op, c;
};
struct RawPass {
  int steps = 0;
  std::vector<RawEntry> e;    // [steps][lanes]
  std::vector<int> lane_len;  // real entries of each lane (the rest of its column is padding)
};

// Lay jobs onto lanes (longest first onto the least loaded lane), then order
// the entries step by step so that the lanes sharing a shared-memory
// wavefront read operands in different banks.  A warp's two operand gathers
// of a step are two shared-memory instructions; each costs as many wavefronts
// as the most distinct addresses any bank receives.  With `width`-byte
// accesses, 128 / width consecutive lanes share a wavefront and the bank key
// of value slot x is x mod (128 / width).  Within a job the entries may come
// in any order (the sum is fixed by the schedule, so still deterministic), and
// with `allow_swap` the two operands of a product may trade places; the
// greedy picks, lane by lane, the entry (among the first kWindow remaining)
// that adds the fewest conflicts, and the last entry of a job carries its
// flush.
RawPass lay_out(const std::vector<Job>& jobs, int lanes, int width, bool allow_swap) {
  constexpr size_t kWindow = 64;
  std::vector<int> order(jobs.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return jobs[x].sides.size() > jobs[y].sides.size(); });
  using LaneLoad = std::pair<size_t, int>;
  std::priority_queue<LaneLoad, std::vector<LaneLoad>, std::greater<LaneLoad>> heap;
  for (int l = 0; l < lanes; ++l) heap.push({0, l});
  std::vector<std::vector<int>> lane_jobs(lanes);
  for (int j : order) {
    auto top = heap.top();
    heap.pop();
    lane_jobs[top.second].push_back(j);
    heap.push({top.first + jobs[j].sides.size(), top.second});
  }
  // longest lanes first, so the short ones share warps that stop early
  // (every warp runs only its own longest lane's steps)
  auto lane_total = [&](const std::vector<int>& js) {
    size_t n = 0;
    for (int j : js) n += jobs[j].sides.size();
    return n;
  };
  std::stable_sort(lane_jobs.begin(), lane_jobs.end(), [&](const std::vector<int>& x, const std::vector<int>& y) {
    return lane_total(x) > lane_total(y);
  });
  RawPass p;
  size_t steps = 0;
  p.lane_len.assign(lanes, 0);
  for (int l = 0; l < lanes; ++l) {
    size_t n = 0;
    for (int j : lane_jobs[l]) n += jobs[j].sides.size();
    steps = std::max(steps, n);
    p.lane_len[l] = static_cast<int>(n);
  }
  p.steps = static_cast<int>(steps);
  p.e.assign(steps * lanes, RawEntry{kSymZero, kSymZero, kSymZero, kOpNone, 0});

  struct LaneState {
    size_t next_job = 0;
    int job = -1;
    std::vector<Side> rem;
  };
  std::vector<LaneState> st(lanes);
  auto advance = [&](int l) {
    LaneState& L = st[l];
    while (L.rem.empty() && L.next_job < lane_jobs[l].size()) {
      L.job = lane_jobs[l][L.next_job++];
      L.rem = jobs[L.job].sides;
    }
    return !L.rem.empty();
  };
  const int group = std::max(1, std::min(32, 128 / std::max(4, width)));
  const uint32_t nkey = static_cast<uint32_t>(group);
  std::vector<std::vector<uint32_t>> usedA(nkey), usedB(nkey);
  auto symbolic = [](uint32_t x) { return x == kSymZero || x == kSymOne; };
  auto load = [&](const std::vector<std::vector<uint32_t>>& used, uint32_t x) -> size_t {
    if (symbolic(x)) return 0;   // one shared constant slot: every lane reads the same address
    const auto& v = used[x % nkey];
    for (uint32_t y : v)
      if (y == x) return 0;
    return v.size();
  };
  auto mark = [&](std::vector<std::vector<uint32_t>>& used, uint32_t x) {
    if (symbolic(x)) return;
    auto& v = used[x % nkey];
    for (uint32_t y : v)
      if (y == x) return;
    v.push_back(x);
  };
  for (size_t s = 0; s < steps; ++s) {
    for (int g0 = 0; g0 < lanes; g0 += group) {
      for (auto& v : usedA) v.clear();
      for (auto& v : usedB) v.clear();
      for (int l = g0; l < std::min(lanes, g0 + group); ++l) {
        if (!advance(l)) continue;   // padding entry (constant-zero slot)
        LaneState& L = st[l];
        size_t best = 0, best_cost = SIZE_MAX;
        bool best_swap = false;
        const size_t ncand = std::min(kWindow, L.rem.size());
        for (size_t i = 0; i < ncand && best_cost > 0; ++i) {
          const Side& c = L.rem[i];
          size_t cost = load(usedA, c.a) + load(usedB, c.b);
          bool sw = false;
          if (allow_swap) {
            const size_t c2 = load(usedA, c.b) + load(usedB, c.a);
            if (c2 < cost) {
              cost = c2;
              sw = true;
            }
          }
          if (cost < best_cost) {
            best_cost = cost;
            best = i;
            best_swap = sw;
          }
        }
        Side c = L.rem[best];
        if (best_swap) std::swap(c.a, c.b);
        L.rem[best] = L.rem.back();
        L.rem.pop_back();
        mark(usedA, c.a);
        mark(usedB, c.b);
        RawEntry& r = p.e[s * lanes + l];
        r.a = c.a;
        r.b = c.b;
        r.c = c.c;
        r.dst = kSymZero;
        r.op = kOpNone;
        if (L.rem.empty()) {
          r.dst = jobs[L.job].dst;
          r.op = jobs[L.job].op;
        }
      }
    }
  }
  return p;
}

// Split long jobs into chunks writing partial slots; returns the main pass and,
// when anything was split, the combine pass.  `parts_used` gets the number of
// partial slots the pass pair needs.
void emit_jobs(const std::vector<Job>& jobs, int lanes, int width, bool allow_swap, std::vector<RawPass>& out,
               int& parts_used) {
  size_t total = 0;
  for (const Job& j : jobs) total += j.sides.size();
  if (total == 0) return;
  size_t cap = std::max<size_t>(4, (total + lanes - 1) / lanes);
  std::vector<Job> main_jobs, comb_jobs;
  int parts = 0;
  for (const Job& j : jobs) {
    if (j.sides.empty()) continue;
    if (j.sides.size() <= cap) {
      main_jobs.push_back(j);
      continue;
    }
    size_t nch = (j.sides.size() + cap - 1) / cap;
    size_t per = (j.sides.size() + nch - 1) / nch;
    Job comb{j.dst, j.op, {}};
    for (size_t c0 = 0; c0 < j.sides.size(); c0 += per) {
      Job ch{kSymPartBase + static_cast<uint32_t>(parts), kOpStore, {}};
      ch.sides.assign(j.sides.begin() + c0, j.sides.begin() + std::min(j.sides.size(), c0 + per));
      main_jobs.push_back(std::move(ch));
      comb.sides.push_back(Side{kSymPartBase + static_cast<uint32_t>(parts), kSymOne, 1});
      ++parts;
    }
    comb_jobs.push_back(std::move(comb));
  }
  out.push_back(lay_out(main_jobs, lanes, width, allow_swap));
  if (!comb_jobs.empty()) out.push_back(lay_out(comb_jobs, lanes, width, false));
  parts_used = std::max(parts_used, parts);
}

}  // namespace

bool adjoint_layout(const Potential& pot, std::vector<int>& dm_pos) {
  const int M = pot.M, B = pot.B;
  dm_pos.resize(M);
  for (int k = 0; k < M; ++k) dm_pos[k] = k;
  if (B == 0) return false;
  int D = 0;
  std::map<std::array<int, 4>, int> basic_of;
  for (int k = 0; k < B; ++k) {
    const int* r = &pot.basic[4 * k];
    D = std::max(D, r[1] + r[2] + r[3]);
    basic_of[{r[0], r[1], r[2], r[3]}] = k;
  }
  std::vector<int> pos(B, -1);
  int next = 0;
  for (int sum = 0; sum <= D; ++sum) {
    for (int a = 0; a <= sum; ++a) {
      const int b = sum - a, top = D - sum;
      for (int k = 0; k <= top; ++k) {
        for (int mu = 0; mu <= k / 2; ++mu) {
          auto it = basic_of.find({mu, a, b, top - k});
          if (it == basic_of.end()) return false;   // a hole: not level-structured
          pos[it->second] = next++;
        }
      }
    }
  }
  if (next != B) return false;                      // basic moments outside the pattern
  for (int k = 0; k < B; ++k) dm_pos[k] = pos[k];
  return true;
}

void seed_list(const Potential& pot, std::vector<int>& idx, std::vector<double>& val) {
  std::map<int, double> acc;
  for (int a = 0; a < pot.Sa; ++a) acc[pot.mapping[a]] += pot.moment[a];
  idx.clear();
  val.clear();
  for (auto& kv : acc) {
    idx.push_back(kv.first);
    val.push_back(kv.second);
  }
}

bool build_schedule(const Potential& pot, int lanes, Schedule& s, std::string& err, int width) {
  s = Schedule();
  s.lanes = lanes;
  s.width = width;
  const int M = pot.M, B = pot.B, T = pot.T;
  if (lanes <= 0 || lanes % 32 != 0) { err = "lanes must be a positive multiple of 32"; return false; }

  // depth of every moment and the write-before-read property
  std::vector<int> depth(M, 0), last_write(M, -1), first_read(M, INT_MAX), is_target(M, 0);
  for (int e = 0; e < T; ++e) {
    const int* r = &pot.times[4 * e];
    if (r[2] < 0 || r[2] >= (1 << 14)) { err = "alpha_index_times multiplicity outside [0, 16383]"; return false; }
    depth[r[3]] = std::max(depth[r[3]], std::max(depth[r[0]], depth[r[1]]) + 1);
    last_write[r[3]] = e;
    is_target[r[3]] = 1;
    first_read[r[0]] = std::min(first_read[r[0]], e);
    first_read[r[1]] = std::min(first_read[r[1]], e);
  }
  for (int k = 0; k < M; ++k) {
    if (last_write[k] >= 0 && first_read[k] <= last_write[k]) {
      err = "alpha_index_times reads a moment before its last contribution; unsupported order";
      return false;
    }
  }
  int maxd = 0;
  for (int k = 0; k < M; ++k) maxd = std::max(maxd, depth[k]);
  s.max_depth = maxd;

  // value-space layout (partials resolved at the end)
  s.v_m = 0;
  s.v_dm = M;
  s.v_part = 2 * M;

  // monomials
  std::map<std::tuple<int, int, int>, int> mono_of;
  std::vector<std::tuple<int, int, int>> monos;
  for (int k = 0; k < B; ++k) {
    auto key = std::make_tuple(pot.basic[4 * k + 1], pot.basic[4 * k + 2], pot.basic[4 * k + 3]);
    if (!mono_of.count(key)) {
      mono_of[key] = static_cast<int>(monos.size());
      monos.push_back(key);
    }
  }
  // degree descending (then a, b, c): the threads of a warp in the basic-moment
  // phase then hold monomials of one degree, i.e. one radial-function count
  std::sort(monos.begin(), monos.end(), [](const std::tuple<int, int, int>& x, const std::tuple<int, int, int>& y) {
    const int dx = std::get<0>(x) + std::get<1>(x) + std::get<2>(x), dy = std::get<0>(y) + std::get<1>(y) + std::get<2>(y);
    return dx != dy ? dx > dy : x < y;
  });
  for (size_t p = 0; p < monos.size(); ++p) mono_of[monos[p]] = static_cast<int>(p);
  s.P = static_cast<int>(monos.size());
  s.mono_abc.assign(4 * s.P, 0);
  s.mono_k.assign(kMaxR * s.P, -1);
  s.D = 0;
  for (int p = 0; p < s.P; ++p) {
    int a, b, c;
    std::tie(a, b, c) = monos[p];
    s.mono_abc[4 * p] = a;
    s.mono_abc[4 * p + 1] = b;
    s.mono_abc[4 * p + 2] = c;
    s.mono_abc[4 * p + 3] = a + b + c;
    s.D = std::max(s.D, a + b + c);
  }
  for (int k = 0; k < B; ++k) {
    int mu = pot.basic[4 * k];
    int p = mono_of[std::make_tuple(pot.basic[4 * k + 1], pot.basic[4 * k + 2], pot.basic[4 * k + 3])];
    if (s.mono_k[kMaxR * p + mu] >= 0) { err = "duplicate row in alpha_index_basic"; return false; }
    s.mono_k[kMaxR * p + mu] = k;
  }
  // radial functions per degree: nmu[v] = 1 + the largest mu of a basic
  // moment of degree v (0 if none)
  s.nmu.assign(s.D + 1, 0);
  for (int k = 0; k < B; ++k) {
    const int v = pot.basic[4 * k + 1] + pot.basic[4 * k + 2] + pot.basic[4 * k + 3];
    s.nmu[v] = std::max(s.nmu[v], pot.basic[4 * k] + 1);
  }
  // dense simplex in pair order
  s.npairs = (s.D + 1) * (s.D + 2) / 2;
  s.Q = (s.D + 1) * (s.D + 2) * (s.D + 3) / 6;
  s.dense_k.assign(static_cast<size_t>(s.Q) * kMaxR, -1);
  {
    int slot = 0;
    for (int sum = 0; sum <= s.D; ++sum) {
      for (int a = 0; a <= sum; ++a) {
        const int b = sum - a;
        for (int c = 0; c <= s.D - sum; ++c, ++slot) {
          auto it = mono_of.find(std::make_tuple(a, b, c));
          if (it == mono_of.end()) continue;
          for (int mu = 0; mu < kMaxR; ++mu)
            s.dense_k[static_cast<size_t>(slot) * kMaxR + mu] = s.mono_k[kMaxR * it->second + mu];
        }
      }
    }
  }
  s.tri = adjoint_layout(pot, s.dm_pos);
  if (s.tri) {
    // pairs (a, b) in pair order with their chain base; longest chain first
    // onto the least loaded warp (cost ~ adjoint loads and multiply-adds of the
    // chain's steps plus its Horner steps and tail)
    struct P3 { int word, cost; };
    std::vector<P3> pairs;
    int base = 0;
    for (int sum = 0; sum <= s.D; ++sum)
      for (int a = 0; a <= sum; ++a) {
        const int b = sum - a, top = s.D - sum;
        int cost = 10;
        for (int k = 0; k <= top; ++k) cost += 3 * (k / 2 + 1) + 3;
        pairs.push_back({a | (b << 4) | (top << 8) | (base << 12), cost});
        base += ((top + 2) * (top + 2)) / 4;
      }
    std::vector<int> order(pairs.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return pairs[x].cost > pairs[y].cost; });
    // one list per group width (kN3GroupWarps: the FP32 kernel; half of it:
    // the FP64 kernel)
    for (int gi = 0; gi < 2; ++gi) {
      const int warps = std::min(lanes / 32, gi == 0 ? kN3GroupWarps : kN3GroupWarps / 2);
      std::vector<std::vector<int>> wl(warps);
      std::vector<long> load(warps, 0);
      for (int i : order) {
        int w = 0;
        for (int v = 1; v < warps; ++v)
          if (load[v] < load[w] || (load[v] == load[w] && wl[v].size() < wl[w].size())) w = v;
        wl[w].push_back(pairs[i].word);
        load[w] += pairs[i].cost;
      }
      std::vector<int>& np = gi == 0 ? s.n3_pairs : s.n3_pairs_half;
      std::vector<int>& no = gi == 0 ? s.n3_off : s.n3_off_half;
      no.assign(1, 0);
      for (int w = 0; w < warps; ++w) {
        if (wl[w].size() > 32) s.tri = false;    // one pair per lane at most
        np.insert(np.end(), wl[w].begin(), wl[w].end());
        no.push_back(static_cast<int>(np.size()));
      }
    }
    if (base >= (1 << 20) || s.D > 15) s.tri = false;
  }
  // moments that are read but never written stay zero for the whole run
  std::vector<char> read(M, 0);
  for (int e = 0; e < T; ++e) { read[pot.times[4 * e]] = 1; read[pot.times[4 * e + 1]] = 1; }
  for (int v : pot.mapping) read[v] = 1;
  for (int k = B; k < M; ++k)
    if (!is_target[k] && read[k]) s.zero_list.push_back(k);

  std::vector<RawPass> fwd, rev;
  int parts = 0;
  // forward: one pass per target depth, jobs = targets in first-appearance order
  for (int L = 1; L <= maxd; ++L) {
    std::vector<Job> jobs;
    std::map<int, int> job_of;
    for (int e = 0; e < T; ++e) {
      const int* r = &pot.times[4 * e];
      if (depth[r[3]] != L) continue;
      auto it = job_of.find(r[3]);
      if (it == job_of.end()) {
        job_of[r[3]] = static_cast<int>(jobs.size());
        jobs.push_back(Job{static_cast<uint32_t>(s.v_m + r[3]), r[3] < B ? kOpAdd : kOpStore, {}});
        it = job_of.find(r[3]);
      }
      jobs[it->second].sides.push_back(
          Side{static_cast<uint32_t>(s.v_m + r[0]), static_cast<uint32_t>(s.v_m + r[1]), static_cast<uint32_t>(r[2])});
    }
    emit_jobs(jobs, lanes, width, true, fwd, parts);
  }
  // reverse: passes for target depth maxd..1 gather sides whose source has
  // depth >= 1; every side into a depth-0 source waits for one final pass.
  // A source's first job in execution order stores its sum unless the slot
  // holds a seed (a scalar moment's coefficient); later ones add to it.
  std::vector<char> seeded(M, 0), written(M, 0);
  for (int v : pot.mapping) seeded[v] = 1;
  auto add_side = [&](std::vector<Job>& jobs, std::map<int, int>& job_of, int src, int tgt, int other, int mult) {
    auto it = job_of.find(src);
    if (it == job_of.end()) {
      job_of[src] = static_cast<int>(jobs.size());
      jobs.push_back(Job{static_cast<uint32_t>(s.v_dm + s.dm_pos[src]),
                         (seeded[src] || written[src]) ? kOpAdd : kOpStore, {}});
      it = job_of.find(src);
    }
    jobs[it->second].sides.push_back(Side{static_cast<uint32_t>(s.v_dm + s.dm_pos[tgt]),
                                          static_cast<uint32_t>(s.v_m + other), static_cast<uint32_t>(mult)});
  };
  for (int L = maxd; L >= 1; --L) {
    std::vector<Job> jobs;
    std::map<int, int> job_of;
    for (int e = 0; e < T; ++e) {
      const int* r = &pot.times[4 * e];
      if (depth[r[3]] != L) continue;
      if (depth[r[0]] >= 1) add_side(jobs, job_of, r[0], r[3], r[1], r[2]);
      if (depth[r[1]] >= 1) add_side(jobs, job_of, r[1], r[3], r[0], r[2]);
    }
    emit_jobs(jobs, lanes, width, false, rev, parts);
    for (const auto& kv : job_of) written[kv.first] = 1;
  }
  {
    std::vector<Job> jobs;
    std::map<int, int> job_of;
    for (int L = maxd; L >= 1; --L) {
      for (int e = 0; e < T; ++e) {
        const int* r = &pot.times[4 * e];
        if (depth[r[3]] != L) continue;
        if (depth[r[0]] == 0) add_side(jobs, job_of, r[0], r[3], r[1], r[2]);
        if (depth[r[1]] == 0) add_side(jobs, job_of, r[1], r[3], r[0], r[2]);
      }
    }
    emit_jobs(jobs, lanes, width, false, rev, parts);
  }
  s.n_part = parts;
  s.v_zero = s.v_part + parts;
  s.v_one = s.v_zero + 1;
  s.v_size = s.v_one + 1;
  if (s.v_size > 65535) { err = "value space above 65535 entries; basis too large"; return false; }
  if (static_cast<int>(fwd.size() + rev.size()) > kMaxPasses * 2) { err = "too many passes"; return false; }

  auto resolve = [&](uint32_t v) -> uint32_t {
    if (v == kSymZero) return static_cast<uint32_t>(s.v_zero);
    if (v == kSymOne) return static_cast<uint32_t>(s.v_one);
    if (v >= kSymPartBase) return static_cast<uint32_t>(s.v_part) + (v - kSymPartBase);
    return v;
  };
  const uint32_t nop_x = static_cast<uint32_t>(s.v_zero) | (static_cast<uint32_t>(s.v_zero) << 16);
  auto push_nops = [&](size_t n) {
    for (size_t i = 0; i < n; ++i) {
      s.entries.push_back(nop_x);
      s.entries.push_back(0u);
    }
  };
  auto flush_passes = [&](std::vector<RawPass>& raw, std::vector<Pass>& dst) {
    for (RawPass& rp : raw) {
      Pass p;
      p.offset = static_cast<int>(s.entries.size() / 2);
      p.steps = (rp.steps + kStepAlign - 1) / kStepAlign * kStepAlign;
      p.wsteps.assign(lanes / 32, 0);
      for (int l = 0; l < lanes; ++l)
        p.wsteps[l / 32] = std::max(p.wsteps[l / 32], (rp.lane_len[l] + kStepAlign - 1) / kStepAlign * kStepAlign);
      for (const RawEntry& r : rp.e) {
        uint32_t a = resolve(r.a), b = resolve(r.b), d = resolve(r.dst);
        s.entries.push_back(a | (b << 16));
        s.entries.push_back(r.c | (r.op << kOpShift) | (d << kDstShift));
      }
      push_nops(static_cast<size_t>(p.steps - rp.steps) * lanes);
      dst.push_back(p);
    }
  };
  flush_passes(fwd, s.fwd);
  flush_passes(rev, s.rev);
  push_nops(static_cast<size_t>(kStepAlign) * lanes);
  // every operand and destination must lie inside the value space
  for (size_t e = 0; e < s.entries.size(); e += 2) {
    const uint32_t x = s.entries[e], y = s.entries[e + 1];
    if ((x & 0xFFFFu) >= static_cast<uint32_t>(s.v_size) || (x >> 16) >= static_cast<uint32_t>(s.v_size) ||
        (y >> kDstShift) >= static_cast<uint32_t>(s.v_size)) {
      err = "internal error: schedule operand outside the value space";
      return false;
    }
  }
  if (static_cast<int>(s.fwd.size()) > kMaxPasses || static_cast<int>(s.rev.size()) > kMaxPasses) {
    err = "too many passes";
    return false;
  }
  return true;
}

namespace {

// Shared-memory wavefronts of one operand gather (x = the a or b field) of the
// lanes [g0, g0 + n) at one step of a pass: the most distinct addresses one
// bank key receives.  The constant slots (zero, one) are read by many lanes at
// once (broadcasts) and count as free.  `hot` gets the lanes whose key has
// that many: only moving one of them can lower the count.
uint32_t gather_wavefronts(const uint32_t* ent, int lanes, size_t row, int g0, int n, bool b_field, uint32_t nkey,
                           uint32_t free0, uint32_t free1, uint32_t* hot) {
  uint32_t addr[32], key_n[32] = {};
  int na = 0;
  for (int i = 0; i < n; ++i) {
    const uint32_t w = ent[2 * (row * lanes + g0 + i)];
    const uint32_t x = b_field ? w >> 16 : w & 0xFFFFu;
    if (x == free0 || x == free1) continue;
    bool seen = false;
    for (int k = 0; k < na && !seen; ++k) seen = addr[k] == x;
    if (!seen) {
      addr[na++] = x;
      ++key_n[x % nkey];
    }
  }
  uint32_t mx = 0;
  for (uint32_t k = 0; k < nkey; ++k) mx = std::max(mx, key_n[k]);
  if (hot) {
    *hot = 0;
    if (mx > 1)
      for (int i = 0; i < n; ++i) {
        const uint32_t w = ent[2 * (row * lanes + g0 + i)];
        const uint32_t x = b_field ? w >> 16 : w & 0xFFFFu;
        if (x != free0 && x != free1 && key_n[x % nkey] == mx) *hot |= 1u << i;
      }
  }
  return mx;
}

}  // namespace

void refine_schedule(Schedule& s) {
  const int lanes = s.lanes;
  const int group = std::max(1, std::min(32, 128 / std::max(4, s.width)));
  const uint32_t nkey = static_cast<uint32_t>(group);
  const uint32_t z = static_cast<uint32_t>(s.v_zero), one = static_cast<uint32_t>(s.v_one);
  constexpr int kTries = 16, kSweeps = 2;
  uint32_t* ent = s.entries.data();
  uint64_t rng = 0x9E3779B97F4A7C15ull;
  auto next = [&]() {
    rng ^= rng << 13;
    rng ^= rng >> 7;
    rng ^= rng << 17;
    return rng;
  };
  auto refine_pass = [&](const Pass& p, bool allow_swap) {
    const size_t steps = static_cast<size_t>(p.steps);
    uint32_t* e = ent + 2 * static_cast<size_t>(p.offset);
    // job spans: a lane's job ends at the entry that flushes; entries after
    // the lane's last flush are padding
    std::vector<int> lo(steps * lanes, 0), hi(steps * lanes, 0);
    for (int l = 0; l < lanes; ++l) {
      size_t start = 0;
      for (size_t t = 0; t < steps; ++t) {
        if (((e[2 * (t * lanes + l) + 1] >> kOpShift) & 3u) == kOpNone) continue;
        for (size_t u = start; u <= t; ++u) {
          lo[u * lanes + l] = static_cast<int>(start);
          hi[u * lanes + l] = static_cast<int>(t + 1);
        }
        start = t + 1;
      }
    }
    auto cost = [&](size_t t, int g0, int n) {
      return gather_wavefronts(e, lanes, t, g0, n, false, nkey, z, one, nullptr) +
             gather_wavefronts(e, lanes, t, g0, n, true, nkey, z, one, nullptr);
    };
    // trade the operands and multiplicity of two entries (flush bits stay)
    auto trade = [&](size_t x, size_t y) {
      std::swap(e[2 * x], e[2 * y]);
      const uint32_t mx = e[2 * x + 1] & kMultMask, my = e[2 * y + 1] & kMultMask;
      e[2 * x + 1] = (e[2 * x + 1] & ~kMultMask) | my;
      e[2 * y + 1] = (e[2 * y + 1] & ~kMultMask) | mx;
    };
    auto flip = [&](size_t x) { e[2 * x] = (e[2 * x] >> 16) | (e[2 * x] << 16); };
    for (int sweep = 0; sweep < kSweeps; ++sweep) {
      size_t gained = 0;
      for (size_t t = 0; t < steps; ++t) {
        for (int g0 = 0; g0 < lanes; g0 += group) {
          const int n = std::min(group, lanes - g0);
          uint32_t hotA, hotB;
          size_t c0 = gather_wavefronts(e, lanes, t, g0, n, false, nkey, z, one, &hotA) +
                      gather_wavefronts(e, lanes, t, g0, n, true, nkey, z, one, &hotB);
          const uint32_t hot = hotA | hotB;
          for (int i = 0; i < n && c0 > 2; ++i) {
            if (!(hot >> i & 1u)) continue;
            const size_t at = t * lanes + g0 + i;
            if (hi[at] == 0) continue;   // padding
            if (allow_swap) {
              flip(at);
              const size_t c1 = cost(t, g0, n);
              if (c1 < c0) {
                gained += c0 - c1;
                c0 = c1;
                continue;
              }
              flip(at);
            }
            const int span = hi[at] - lo[at];
            if (span < 2) continue;
            for (int k = 0; k < kTries; ++k) {
              const size_t t2 = static_cast<size_t>(lo[at]) + next() % static_cast<uint64_t>(span);
              if (t2 == t) continue;
              const size_t at2 = t2 * lanes + g0 + i;
              const size_t before = c0 + cost(t2, g0, n);
              trade(at, at2);
              const size_t c1 = cost(t, g0, n), after = c1 + cost(t2, g0, n);
              if (after < before) {
                gained += before - after;
                c0 = c1;
                break;
              }
              trade(at, at2);
            }
          }
        }
      }
      if (gained == 0) break;
    }
  };
  for (const Pass& p : s.fwd) refine_pass(p, true);
  for (const Pass& p : s.rev) refine_pass(p, false);
}

double emulate_schedule(const Potential& pot, const Schedule& s, std::vector<double>& V) {
  V.resize(s.v_size, 0.0);
  for (int k : s.zero_list) V[s.v_m + k] = 0.0;
  V[s.v_zero] = 0.0;
  V[s.v_one] = 1.0;
  auto run = [&](const Pass& p) {
    // Lanes run one after another: the schedule guarantees that no lane reads
    // a slot another lane writes in the same pass, so this equals the device.
    std::vector<double> out;
    std::vector<std::pair<int, std::pair<int, double>>> writes;
    for (int l = 0; l < s.lanes; ++l) {
      double acc = 0.0;
      // a warp runs only its own step count (Pass::wsteps), as on the device
      for (int st = 0; st < p.wsteps[l / 32]; ++st) {
        size_t e = static_cast<size_t>(p.offset) + static_cast<size_t>(st) * s.lanes + l;
        uint32_t x = s.entries[2 * e], y = s.entries[2 * e + 1];
        int a = x & 0xFFFF, b = x >> 16, d = y >> kDstShift, op = (y >> kOpShift) & 3;
        double c = static_cast<double>(y & kMultMask);
        acc = std::fma(c * V[a], V[b], acc);
        if (op != kOpNone) {
          writes.push_back({d, {static_cast<int>(op), acc}});
          acc = 0.0;
        }
      }
    }
    for (auto& w : writes) {
      if (w.second.first == kOpStore) V[w.first] = w.second.second;
      else V[w.first] += w.second.second;
    }
  };
  for (const Pass& p : s.fwd) run(p);
  double e = 0.0;
  for (int a = 0; a < pot.Sa; ++a) e += pot.moment[a] * V[s.v_m + pot.mapping[a]];
  for (int k = 0; k < pot.M; ++k) V[s.v_dm + k] = 0.0;
  std::vector<int> si;
  std::vector<double> sv;
  seed_list(pot, si, sv);
  for (size_t i = 0; i < si.size(); ++i) V[s.v_dm + s.dm_pos[si[i]]] = sv[i];
  for (const Pass& p : s.rev) run(p);
  return e;
}

}  // namespace mtp
