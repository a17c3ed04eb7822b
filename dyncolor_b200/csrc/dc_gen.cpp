// dc_gen.cpp -- seeded synthetic workload generators (include/dyncolor_gen.h).
//
// Random numbers: SplitMix64 (Steele, Lea, Flood 2014), one stream per
// sample index for the bulk generators so results do not depend on the
// number of OpenMP threads.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/dyncolor_gen.h"

namespace {

inline uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

inline uint64_t stream_seed(uint64_t seed, uint64_t i) {
  uint64_t x = seed ^ (i * 0xd1b54a32d192ed03ull);
  return splitmix64(x);
}

struct RmatThresholds {
  uint64_t ta, tab, tabc;  // cumulative quadrant probabilities scaled to 2^32
};

RmatThresholds rmat_thresholds(double a, double b, double c) {
  const double s = 4294967296.0;
  RmatThresholds t;
  t.ta = (uint64_t)(a * s);
  t.tab = (uint64_t)((a + b) * s);
  t.tabc = (uint64_t)((a + b + c) * s);
  return t;
}

inline void rmat_pair(uint64_t& x, int scale, const RmatThresholds& t, uint64_t& u, uint64_t& v) {
  u = 0;
  v = 0;
  uint64_t r = 0;
  for (int l = 0; l < scale; ++l) {
    if ((l & 1) == 0) r = splitmix64(x);
    const uint64_t q = (l & 1) ? (r >> 32) : (r & 0xffffffffull);
    const uint64_t bit = 1ull << (scale - 1 - l);
    if (q < t.ta) {
    } else if (q < t.tab) {
      v |= bit;
    } else if (q < t.tabc) {
      u |= bit;
    } else {
      u |= bit;
      v |= bit;
    }
  }
}

inline uint64_t uniform_below(uint64_t& x, uint64_t n) {
  // multiply-shift reduction of a 64-bit draw
  return (uint64_t)(((unsigned __int128)splitmix64(x) * n) >> 64);
}

// Parallel LSD radix sort of 64-bit keys, 16-bit digits; stable per pass.
void radix_sort_u64(uint64_t* a, int64_t n) {
  if (n <= 1) return;
  std::vector<uint64_t> tmp((size_t)n);
  uint64_t* src = a;
  uint64_t* dst = tmp.data();
  const int nt = std::max(1, omp_get_max_threads());
  std::vector<int64_t> hist((size_t)nt * 65536);
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = pass * 16;
    std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
      int64_t* h = &hist[(size_t)t * 65536];
      for (int64_t i = lo; i < hi; ++i) ++h[(src[i] >> shift) & 0xffff];
    }
    bool skip = false;
    int64_t run = 0;
    for (int d = 0; d < 65536; ++d) {
      int64_t tot = 0;
      for (int t = 0; t < nt; ++t) tot += hist[(size_t)t * 65536 + d];
      if (tot == n) skip = true;
      for (int t = 0; t < nt; ++t) {
        const int64_t x = hist[(size_t)t * 65536 + d];
        hist[(size_t)t * 65536 + d] = run;
        run += x;
      }
    }
    if (skip) continue;
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
      int64_t* h = &hist[(size_t)t * 65536];
      for (int64_t i = lo; i < hi; ++i) dst[h[(src[i] >> shift) & 0xffff]++] = src[i];
    }
    std::swap(src, dst);
  }
  if (src != a) std::memcpy(a, src, (size_t)n * sizeof(uint64_t));
}

inline uint64_t pair_key(int32_t u, int32_t v) {
  const uint32_t lo = (uint32_t)std::min(u, v), hi = (uint32_t)std::max(u, v);
  return ((uint64_t)lo << 32) | hi;
}

// Open-addressing set of 64-bit keys (EMPTY = all ones).
struct KeySet {
  std::vector<uint64_t> slot;
  int64_t count = 0;
  static constexpr uint64_t EMPTY = ~0ull;
  void init(int64_t cap) {
    int64_t c = 16;
    while (c < 2 * cap) c <<= 1;
    slot.assign((size_t)c, EMPTY);
    count = 0;
  }
  static uint64_t hash(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return k;
  }
  bool contains(uint64_t k) const {
    const uint64_t mask = slot.size() - 1;
    for (uint64_t h = hash(k) & mask;; h = (h + 1) & mask) {
      if (slot[h] == k) return true;
      if (slot[h] == EMPTY) return false;
    }
  }
  bool insert(uint64_t k) {
    if (2 * (count + 1) > (int64_t)slot.size()) grow();
    const uint64_t mask = slot.size() - 1;
    for (uint64_t h = hash(k) & mask;; h = (h + 1) & mask) {
      if (slot[h] == k) return false;
      if (slot[h] == EMPTY) {
        slot[h] = k;
        ++count;
        return true;
      }
    }
  }
  void grow() {
    std::vector<uint64_t> old;
    old.swap(slot);
    slot.assign(old.size() * 2, EMPTY);
    count = 0;
    for (uint64_t k : old)
      if (k != EMPTY) insert(k);
  }
};

}  // namespace

struct dcg_edgeset {
  int32_t n = 0;
  std::vector<uint64_t> e0;  // sorted keys of the original edges
  std::vector<uint8_t> dead;
  int64_t ndead = 0;
  KeySet ins;  // inserted since creation (never deleted by the sampler)
  uint64_t draws = 0;

  bool present(uint64_t k) const {
    auto it = std::lower_bound(e0.begin(), e0.end(), k);
    if (it != e0.end() && *it == k && !dead[(size_t)(it - e0.begin())]) return true;
    return ins.contains(k);
  }
};

extern "C" {

int dcg_rmat(int32_t scale, int32_t n, int64_t m, double a, double b, double c, uint64_t seed,
             int32_t* out_a, int32_t* out_b) {
  if (scale < 1 || scale > 31 || m < 0 || n <= 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return DC_E_INVAL;
  const RmatThresholds t = rmat_thresholds(a, b, c);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    uint64_t x = stream_seed(seed, (uint64_t)i);
    uint64_t u, v;
    rmat_pair(x, scale, t, u, v);
    out_a[i] = (int32_t)(u % (uint64_t)n);
    out_b[i] = (int32_t)(v % (uint64_t)n);
  }
  return DC_OK;
}

int dcg_uniform_pairs(int32_t n, int64_t m, uint64_t seed, int32_t* out_a, int32_t* out_b) {
  if (n <= 0 || m < 0) return DC_E_INVAL;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    uint64_t x = stream_seed(seed, (uint64_t)i);
    out_a[i] = (int32_t)uniform_below(x, (uint64_t)n);
    out_b[i] = (int32_t)uniform_below(x, (uint64_t)n);
  }
  return DC_OK;
}

int64_t dcg_chung_lu(int32_t n, double gamma, double avg_deg, double max_deg, uint64_t seed,
                     int32_t* out_a, int32_t* out_b, int64_t m_cap) {
  if (n <= 1 || gamma <= 1.0 || avg_deg <= 0 || max_deg < avg_deg) return -DC_E_INVAL;
  const double alpha = 1.0 / (gamma - 1.0);
  // mean weight as a function of i0 is increasing: bisection on log(i0)
  auto mean_w = [&](double i0) {
    double s = 0;
    for (int32_t i = 0; i < n; ++i) s += max_deg * std::pow(1.0 + i / i0, -alpha);
    return s / n;
  };
  double lo = 1e-6, hi = (double)n * 1e3;
  for (int it = 0; it < 100; ++it) {
    const double mid = std::sqrt(lo * hi);
    if (mean_w(mid) < avg_deg)
      lo = mid;
    else
      hi = mid;
  }
  const double i0 = std::sqrt(lo * hi);
  std::vector<double> cdf((size_t)n);
  double acc = 0;
  for (int32_t i = 0; i < n; ++i) {
    acc += max_deg * std::pow(1.0 + i / i0, -alpha);
    cdf[(size_t)i] = acc;
  }
  const int64_t m = std::min<int64_t>((int64_t)std::llround((double)n * avg_deg / 2.0), m_cap);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    uint64_t x = stream_seed(seed, (uint64_t)i);
    const double r1 = (double)(splitmix64(x) >> 11) * 0x1.0p-53 * acc;
    const double r2 = (double)(splitmix64(x) >> 11) * 0x1.0p-53 * acc;
    out_a[i] = (int32_t)std::min<int64_t>(std::upper_bound(cdf.begin(), cdf.end(), r1) - cdf.begin(), n - 1);
    out_b[i] = (int32_t)std::min<int64_t>(std::upper_bound(cdf.begin(), cdf.end(), r2) - cdf.begin(), n - 1);
  }
  return m;
}

int64_t dcg_dedup(int32_t n, int32_t* a, int32_t* b, int64_t m) {
  (void)n;
  std::vector<uint64_t> keys;
  try {
    keys.resize((size_t)m);
  } catch (...) {
    return -DC_E_NOMEM;
  }
  int64_t w = 0;
  // drop self-loops while packing (order preserved)
  for (int64_t i = 0; i < m; ++i)
    if (a[i] != b[i]) keys[(size_t)w++] = pair_key(a[i], b[i]);
  keys.resize((size_t)w);
  radix_sort_u64(keys.data(), w);
  int64_t u = 0;
  for (int64_t i = 0; i < w; ++i) {
    if (i > 0 && keys[(size_t)i] == keys[(size_t)i - 1]) continue;
    a[u] = (int32_t)(keys[(size_t)i] >> 32);
    b[u] = (int32_t)(keys[(size_t)i] & 0xffffffffull);
    ++u;
  }
  return u;
}

int dcg_greedy_color(int32_t n, const int32_t* a, const int32_t* b, int64_t m, int32_t* colors) {
  if (n < 0 || m < 0) return DC_E_INVAL;
  std::vector<int64_t> off((size_t)n + 1, 0);
  for (int64_t i = 0; i < m; ++i) {
    if (a[i] == b[i]) continue;
    ++off[(size_t)std::max(a[i], b[i]) + 1];
  }
  for (int32_t v = 0; v < n; ++v) off[(size_t)v + 1] += off[(size_t)v];
  std::vector<int32_t> lower((size_t)std::max<int64_t>(off[(size_t)n], 1));
  std::vector<int64_t> cur(off.begin(), off.end() - 1);
  for (int64_t i = 0; i < m; ++i) {
    if (a[i] == b[i]) continue;
    const int32_t hi = std::max(a[i], b[i]), lo = std::min(a[i], b[i]);
    lower[(size_t)cur[(size_t)hi]++] = lo;
  }
  std::vector<uint32_t> stamp;
  uint32_t gen = 0;
  for (int32_t v = 0; v < n; ++v) {
    const int64_t L = off[(size_t)v + 1] - off[(size_t)v];
    if ((int64_t)stamp.size() < L + 2) stamp.resize((size_t)(L + 2) * 2, 0);
    ++gen;
    for (int64_t i = off[(size_t)v]; i < off[(size_t)v + 1]; ++i) {
      const int32_t c = colors[lower[(size_t)i]];
      if (c <= L) stamp[(size_t)c] = gen;
    }
    int32_t c = 0;
    while (stamp[(size_t)c] == gen) ++c;
    colors[v] = c;
  }
  return DC_OK;
}

dcg_edgeset* dcg_edgeset_create(int32_t n, const int32_t* a, const int32_t* b, int64_t m) {
  dcg_edgeset* s = new (std::nothrow) dcg_edgeset();
  if (!s) return nullptr;
  try {
    s->n = n;
    s->e0.resize((size_t)m);
    for (int64_t i = 0; i < m; ++i) s->e0[(size_t)i] = pair_key(a[i], b[i]);
    radix_sort_u64(s->e0.data(), m);
    s->e0.erase(std::unique(s->e0.begin(), s->e0.end()), s->e0.end());
    s->dead.assign(s->e0.size(), 0);
    s->ins.init(1024);
  } catch (...) {
    delete s;
    return nullptr;
  }
  return s;
}

void dcg_edgeset_destroy(dcg_edgeset* s) { delete s; }

int64_t dcg_edgeset_size(const dcg_edgeset* s) {
  return (int64_t)s->e0.size() - s->ndead + s->ins.count;
}

int64_t dcg_edgeset_sample_batch(dcg_edgeset* s, int64_t k_del, int64_t k_ins, int32_t ins_mode,
                                 int32_t scale, double a, double b, double c, uint64_t seed,
                                 dc_change* out) {
  if (!s || k_del < 0 || k_ins < 0 || s->n < 2) return -DC_E_INVAL;
  const int64_t alive0 = (int64_t)s->e0.size() - s->ndead;
  if (k_del > alive0) return -DC_E_INVAL;
  uint64_t x = stream_seed(seed, 0x5eed0000ull + s->draws++);
  int64_t w = 0;
  const uint64_t E = s->e0.size();
  // pairs deleted by this batch may not be re-inserted by it: inside one
  // batch a deletion wins over an insertion of the same edge
  KeySet deleted_now;
  deleted_now.init(k_del + 16);
  for (int64_t d = 0; d < k_del; ++d) {
    for (;;) {
      const uint64_t i = uniform_below(x, E);
      if (s->dead[i]) continue;
      s->dead[i] = 1;
      ++s->ndead;
      deleted_now.insert(s->e0[i]);
      out[w].node1 = (int32_t)(s->e0[i] >> 32);
      out[w].node2 = (int32_t)(s->e0[i] & 0xffffffffull);
      out[w].inst = 0;
      ++w;
      break;
    }
  }
  const RmatThresholds t = rmat_thresholds(a, b, c);
  const uint64_t n = (uint64_t)s->n;
  // Candidates are drawn and membership-checked in parallel (one random
  // stream per candidate index), then accepted in index order, so the
  // result does not depend on the thread count.
  const uint64_t round_seed = splitmix64(x);
  int64_t need = k_ins, drawn = 0;
  std::vector<uint64_t> cand;
  std::vector<uint8_t> ok;
  while (need > 0) {
    if (drawn > 1000 * (k_ins + 16)) return -DC_E_INVAL;  // graph too dense for the request
    const int64_t C = need + need / 8 + 64;
    cand.assign((size_t)C, 0);
    ok.assign((size_t)C, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < C; ++i) {
      uint64_t y = stream_seed(round_seed, (uint64_t)(drawn + i));
      uint64_t u = 0, v = 0;
      if (ins_mode == DCG_INS_RMAT) {
        rmat_pair(y, scale, t, u, v);
        u %= n;
        v %= n;
      } else if (ins_mode == DCG_INS_DEGREE && E > 0) {
        const uint64_t j = uniform_below(y, E);
        u = (splitmix64(y) & 1) ? (s->e0[j] >> 32) : (s->e0[j] & 0xffffffffull);
        v = uniform_below(y, n);
      } else {
        u = uniform_below(y, n);
        v = uniform_below(y, n);
      }
      if (u == v) continue;
      const uint64_t k = pair_key((int32_t)u, (int32_t)v);
      cand[(size_t)i] = k;
      ok[(size_t)i] = !s->present(k);
    }
    drawn += C;
    for (int64_t i = 0; i < C && need > 0; ++i) {
      if (!ok[(size_t)i]) continue;
      const uint64_t k = cand[(size_t)i];
      if (deleted_now.contains(k) || !s->ins.insert(k)) continue;
      // randomise which endpoint is node1
      const bool flip = (k ^ (k >> 29)) & 1;
      out[w].node1 = (int32_t)(flip ? (k & 0xffffffffull) : (k >> 32));
      out[w].node2 = (int32_t)(flip ? (k >> 32) : (k & 0xffffffffull));
      out[w].inst = 1;
      ++w;
      --need;
    }
  }
  for (int64_t i = w - 1; i > 0; --i) {
    const int64_t j = (int64_t)uniform_below(x, (uint64_t)i + 1);
    std::swap(out[i], out[j]);
  }
  return w;
}

}  // extern "C"
