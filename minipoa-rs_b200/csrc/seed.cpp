// Seed windows for seeded alignment, restating src/minimizer.rs:28-503 of
// minipoa-rs (repeat filter, exact anchors, sparse chaining, window
// partition). Minimizer selection is this library's own: the reference takes
// it from the simd-minimizers crate (=3.0.0, not vendored), so which k-mer of
// a window is chosen can differ; the k-mer values, the run splitting at
// ambiguous symbols and everything after the sketch follow the reference.
#include "seed.h"

#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <unordered_map>

namespace poa {
namespace {

bool is_base(uint8_t c) {
  const uint8_t u = uint8_t(c & ~0x20);  // ASCII upper case
  return u == 'A' || u == 'C' || u == 'G' || u == 'T' || u == 'U';
}

// 2-bit code of a DNA letter as packed sequences store it: (ASCII >> 1) & 3
// gives A0 C1 T2 G3 for either case, and U packs as T.
uint64_t pack2(uint8_t c) { return (uint64_t(c) >> 1) & 3u; }

// Forward ntHash (Mohamadi et al., Bioinformatics 32:3492, 2016): one random
// 64-bit seed per base, h(k-mer) = XOR over i of rol(seed[b_i], k - 1 - i),
// updated by one rotation per step. Minimizers are ranked by this hash.
constexpr uint64_t kSeed[4] = {0x3c8bfbb395c60474ull, 0x3193c18562a02b4cull, 0x295549f54be24456ull,
                               0x20323ed082572324ull};  // A, C, T, G (2-bit order)
inline uint64_t rol(uint64_t x, unsigned r) {
  r &= 63u;
  return r ? (x << r) | (x >> (64u - r)) : x;
}

}  // namespace

// sketch (src/minimizer.rs:39-75): forward minimizers per run of DNA letters;
// a run shorter than k gives none, and a run with fewer than w k-mers is one
// window of all of them. Leftmost k-mer of smallest hash per window; each
// chosen k-mer is reported once.
std::vector<Minimizer> sketch(const uint8_t *seq, int64_t len, int64_t k, int64_t w) {
  std::vector<Minimizer> out;
  if (k < 1 || k > 31 || w < 1 || w >= 32768 || len >= int64_t(UINT32_MAX)) return out;
  int64_t start = 0;
  std::vector<uint64_t> hash, value;
  while (start < len) {
    while (start < len && !is_base(seq[start])) ++start;
    int64_t end = start;
    while (end < len && is_base(seq[end])) ++end;
    const int64_t n = end - start;
    if (n >= k) {
      const int64_t nk = n - k + 1;
      hash.assign(size_t(nk), 0);
      value.assign(size_t(nk), 0);
      uint64_t h = 0, v = 0;
      const uint64_t vmask = k == 32 ? ~0ull : ((1ull << (2 * k)) - 1);
      for (int64_t i = 0; i < n; ++i) {
        const uint64_t b = pack2(seq[start + i]);
        v = ((v >> 2) | (b << (2 * (k - 1)))) & vmask;  // first base in the low bits
        if (i < k) {
          h = rol(h, 1) ^ kSeed[b];
        } else {
          const uint64_t out_b = pack2(seq[start + i - k]);
          h = rol(h, 1) ^ rol(kSeed[out_b], unsigned(k)) ^ kSeed[b];
        }
        if (i >= k - 1) {
          hash[size_t(i - k + 1)] = h;
          value[size_t(i - k + 1)] = v;
        }
      }
      const int64_t win = std::min<int64_t>(w, nk);
      std::deque<int64_t> dq;  // increasing hashes; front = leftmost minimum
      int64_t last = -1;
      for (int64_t i = 0; i < nk; ++i) {
        while (!dq.empty() && hash[size_t(dq.back())] > hash[size_t(i)]) dq.pop_back();
        dq.push_back(i);
        if (dq.front() <= i - win) dq.pop_front();
        if (i >= win - 1 && dq.front() != last) {
          last = dq.front();
          out.push_back(Minimizer{value[size_t(last)], start + last + k - 1, k});
        }
      }
    }
    start = end + 1;
  }
  return out;
}

// repeat_intervals (src/minimizer.rs:79-110): a seed seen again within
// max_dist marks [previous start - period, end + 1 + period) as tandem
// repeat; intervals closer than 50 bases merge.
std::vector<std::pair<int64_t, int64_t>> repeat_intervals(const std::vector<Minimizer> &mm, int64_t len,
                                                          int64_t max_dist) {
  std::vector<std::pair<int64_t, int64_t>> merged;
  if (max_dist == 0) return merged;
  std::unordered_map<uint64_t, int64_t> last;
  std::vector<std::pair<int64_t, int64_t>> iv;
  for (const Minimizer &s : mm) {
    auto it = last.find(s.value);
    if (it != last.end()) {
      const int64_t previous = it->second;
      const int64_t period = std::max<int64_t>(s.end - previous, 0);
      if (period > 0 && period <= max_dist) {
        const int64_t a = std::max<int64_t>(std::max<int64_t>(previous + 1 - s.span, 0) - period, 0);
        const int64_t b = std::min<int64_t>(s.end + 1 + period, len);
        iv.emplace_back(a, b);
      }
      it->second = s.end;
    } else {
      last.emplace(s.value, s.end);
    }
  }
  std::sort(iv.begin(), iv.end());
  for (auto &x : iv) {
    if (!merged.empty() && x.first <= merged.back().second + 50) {
      merged.back().second = std::max(merged.back().second, x.second);
      continue;
    }
    merged.push_back(x);
  }
  return merged;
}

namespace {

std::vector<int64_t> repeat_coverage(const std::vector<Minimizer> &mm, int64_t len, int64_t max_dist) {
  std::vector<int64_t> prefix(size_t(len) + 1, 0);
  for (auto &x : repeat_intervals(mm, len, max_dist))
    for (int64_t i = x.first + 1; i <= x.second; ++i) prefix[size_t(i)] = 1;
  for (int64_t i = 0; i < len; ++i) prefix[size_t(i) + 1] += prefix[size_t(i)];
  return prefix;
}

bool overlaps_repeat(const Minimizer &m, const std::vector<int64_t> &prefix) {
  return prefix[size_t(m.end + 1)] > prefix[size_t(m.end + 1 - m.span)];
}

// chain_score (src/minimizer.rs:174-193): nothing when b is not before a on
// the query, or more than 1000 query bases before it.
bool chain_score(const Anchor &a, const Anchor &b, int64_t k, int32_t *out) {
  if (a.query_end < b.query_end || a.target_end < b.target_end) return false;
  const int64_t dq = a.query_end - b.query_end, dr = a.target_end - b.target_end;
  if (dq == 0 || dq > 1000) return false;
  const int64_t delta = dr > dq ? dr - dq : dq - dr;
  const int64_t distance = std::min(dr, dq);
  int32_t score = int32_t(std::min(a.span, distance));
  if (delta > 0 || distance > a.span) {
    if (dr == 0) {
      score += 1;
    } else {
      const double linear = 0.01 * double(k) * double(delta);
      const double logarithmic = std::log2(double(delta + 1));
      score -= int32_t(std::min(linear, logarithmic));
    }
  }
  *out = score;
  return true;
}

}  // namespace

// collect_anchors (src/minimizer.rs:128-172): exact forward matches of query
// and target minimizers outside tandem repeats, dropping values that occur
// more than max_occ times on either side; sorted by (target, query), unique.
std::vector<Anchor> collect_anchors(const HostParams &p, const uint8_t *q, int64_t qlen, const uint8_t *t,
                                    int64_t tlen) {
  std::vector<Anchor> anchors;
  if (p.alphabet.size() > 5) return anchors;
  const auto qmm = sketch(q, qlen, int64_t(p.k), int64_t(p.w));
  const auto tmm = sketch(t, tlen, int64_t(p.k), int64_t(p.w));
  const auto qcov = repeat_coverage(qmm, qlen, int64_t(p.tr_dist));
  const auto tcov = repeat_coverage(tmm, tlen, int64_t(p.tr_dist));
  std::map<uint64_t, std::vector<Minimizer>> qindex, tindex;
  for (auto &m : qmm) qindex[m.value].push_back(m);
  for (auto &m : tmm) tindex[m.value].push_back(m);
  for (auto &kv : tindex) {
    auto it = qindex.find(kv.first);
    if (it == qindex.end()) continue;
    if (p.max_occ > 0 && (kv.second.size() > p.max_occ || it->second.size() > p.max_occ)) continue;
    for (auto &tm : kv.second) {
      if (overlaps_repeat(tm, tcov)) continue;
      for (auto &qm : it->second) {
        if (overlaps_repeat(qm, qcov)) continue;
        anchors.push_back(Anchor{tm.end, qm.end, int64_t(p.k), false});
      }
    }
  }
  std::sort(anchors.begin(), anchors.end(), [](const Anchor &a, const Anchor &b) {
    return a.target_end != b.target_end ? a.target_end < b.target_end : a.query_end < b.query_end;
  });
  anchors.erase(std::unique(anchors.begin(), anchors.end()), anchors.end());
  return anchors;
}

// chain (src/minimizer.rs:199-366): sparse chaining over a 1000-base horizon
// (at most 5000 predecessors, 50 non-improving and 25 skipped candidates),
// local chains of >= 3 seeds scoring >= 100, then a DP joining local chains;
// the result is strictly increasing on both sequences.
std::vector<Anchor> chain(const std::vector<Anchor> &anchors, int64_t k) {
  std::vector<Anchor> monotone;
  if (anchors.empty()) return monotone;
  const int64_t n = int64_t(anchors.size());
  std::vector<int32_t> scores(size_t(n), 0);
  std::vector<int64_t> parent(size_t(n), -1);
  std::vector<int64_t> touched(size_t(n), -1);
  int64_t start = 0;
  for (int64_t i = 0; i < n; ++i) {
    while (start < i && std::max<int64_t>(anchors[size_t(i)].target_end - anchors[size_t(start)].target_end, 0) > 1000)
      ++start;
    start = std::max<int64_t>(start, std::max<int64_t>(i - 5000, 0));
    int32_t best = int32_t(anchors[size_t(i)].span);
    int64_t skip = 0, iterations = 0;
    for (int64_t j = i - 1; j >= start; --j) {
      int32_t step = 0;
      if (!chain_score(anchors[size_t(i)], anchors[size_t(j)], k, &step)) continue;
      const int32_t candidate = step + scores[size_t(j)];
      if (candidate > best) {
        best = candidate;
        parent[size_t(i)] = j;
        skip = std::max<int64_t>(skip - 1, 0);
      } else {
        if (candidate != best) {
          if (++iterations > 50) break;
        }
        if (touched[size_t(j)] == i) {
          if (++skip > 25) break;
        }
      }
      if (parent[size_t(j)] >= 0) touched[size_t(parent[size_t(j)])] = i;
    }
    scores[size_t(i)] = best;
  }
  std::vector<char> has_child(size_t(n), 0);
  for (int64_t p : parent)
    if (p >= 0) has_child[size_t(p)] = 1;
  std::vector<int64_t> terminals;
  for (int64_t i = 0; i < n; ++i)
    if (!has_child[size_t(i)] && scores[size_t(i)] >= 100) terminals.push_back(i);
  std::sort(terminals.begin(), terminals.end(), [&](int64_t a, int64_t b) {
    return scores[size_t(a)] != scores[size_t(b)] ? scores[size_t(a)] < scores[size_t(b)] : a < b;
  });
  std::vector<char> used(size_t(n), 0);
  std::vector<std::vector<int64_t>> locals;
  for (auto it = terminals.rbegin(); it != terminals.rend(); ++it) {
    const int64_t end = *it;
    if (used[size_t(end)]) continue;
    int64_t current = end;
    std::vector<int64_t> indexes;
    int32_t best_gain = 0;
    int64_t best_cut = -1;
    while (current >= 0) {
      const int64_t i = current;
      if (used[size_t(i)]) break;
      indexes.push_back(i);
      current = parent[size_t(i)];
      const int32_t gain = scores[size_t(end)] - (current >= 0 ? scores[size_t(current)] : 0);
      if (gain > best_gain) {
        best_gain = gain;
        best_cut = current;
      } else if (best_gain - gain > 1000) {
        current = best_cut;
        break;
      }
    }
    if (current >= 0)
      while (!indexes.empty() && indexes.back() <= current) indexes.pop_back();
    for (int64_t i : indexes) used[size_t(i)] = 1;
    const int32_t local_score = scores[size_t(end)] - (current >= 0 ? scores[size_t(current)] : 0);
    if (indexes.size() >= 3 && local_score >= 100) {
      std::reverse(indexes.begin(), indexes.end());
      locals.push_back(std::move(indexes));
    }
  }
  if (locals.empty()) return monotone;
  std::sort(locals.begin(), locals.end(), [&](const std::vector<int64_t> &a, const std::vector<int64_t> &b) {
    const Anchor &x = anchors[size_t(a.back())], &y = anchors[size_t(b.back())];
    return x.target_end != y.target_end ? x.target_end < y.target_end : x.query_end < y.query_end;
  });
  const size_t L = locals.size();
  std::vector<int32_t> totals(L, 0);
  std::vector<int64_t> previous(L, -1);
  std::vector<size_t> trim(L, 0);
  for (size_t i = 0; i < L; ++i) {
    const auto &local = locals[i];
    std::vector<int32_t> prefix(local.size(), int32_t(anchors[size_t(local[0])].span));
    for (size_t x = 1; x < local.size(); ++x) {
      int32_t step = 0;
      if (!chain_score(anchors[size_t(local[x])], anchors[size_t(local[x - 1])], k, &step)) step = 0;
      prefix[x] = prefix[x - 1] + step;
    }
    totals[i] = prefix.back();
    const Anchor &first = anchors[size_t(local[0])];
    for (size_t jj = i; jj-- > 0;) {
      if (first.target_end < anchors[size_t(locals[jj][0])].target_end) continue;
      const Anchor &last = anchors[size_t(locals[jj].back())];
      size_t offset = local.size();
      for (size_t v = 0; v < local.size(); ++v) {
        const Anchor &a = anchors[size_t(local[v])];
        if (a.target_end > last.target_end && a.query_end > last.query_end) {
          offset = v;
          break;
        }
      }
      if (offset == local.size()) continue;
      const int32_t remaining = prefix.back() - prefix[offset] + int32_t(anchors[size_t(local[offset])].span);
      const int32_t candidate = totals[jj] + remaining;
      if (candidate > totals[i]) {
        totals[i] = candidate;
        previous[i] = int64_t(jj);
        trim[i] = offset;
      }
    }
  }
  // largest total, the lowest index on ties
  size_t best = 0;
  for (size_t i = 1; i < L; ++i)
    if (totals[i] > totals[best]) best = i;
  std::vector<size_t> ids;
  for (int64_t nx = int64_t(best); nx >= 0; nx = previous[size_t(nx)]) ids.push_back(size_t(nx));
  std::reverse(ids.begin(), ids.end());
  for (size_t i : ids)
    for (size_t v = trim[i]; v < locals[i].size(); ++v) {
      const Anchor &a = anchors[size_t(locals[i][v])];
      if (monotone.empty() || (a.target_end > monotone.back().target_end && a.query_end > monotone.back().query_end))
        monotone.push_back(a);
    }
  return monotone;
}

// partition_windows (src/minimizer.rs:371-457): window boundaries along the
// chain by cumulative diagonal drift, seed spacing and maximum window length;
// a boundary forced past those limits marks the window before it adaptive.
std::pair<std::vector<Anchor>, bool> partition_windows(const std::vector<Anchor> &ch, int64_t tlen, int64_t qlen,
                                                       int64_t max_drift, int64_t max_win) {
  const int64_t n = int64_t(ch.size());
  auto te = [&](int64_t i) -> int64_t { return i < 0 ? -1 : ch[size_t(i)].target_end; };
  auto qe = [&](int64_t i) -> int64_t { return i < 0 ? -1 : ch[size_t(i)].query_end; };
  auto ts = [&](int64_t i) -> int64_t { return i == n ? tlen : ch[size_t(i)].target_end - ch[size_t(i)].span + 1; };
  auto qs = [&](int64_t i) -> int64_t { return i == n ? qlen : ch[size_t(i)].query_end - ch[size_t(i)].span + 1; };
  auto diag = [&](int64_t i) -> int64_t {
    if (i < 0) return 0;
    if (i == n) return tlen - qlen;
    return te(i) - qe(i);
  };
  auto absd = [](int64_t x) -> uint64_t { return x < 0 ? uint64_t(-x) : uint64_t(x); };
  std::vector<Anchor> selected;
  bool tail = false;
  int64_t s = -1;
  while (s < n) {
    int64_t boundary = -1;
    for (int64_t i = s + 1; i <= n; ++i) {
      const int64_t gt = ts(i) - te(s) - 1, gq = qs(i) - qe(s) - 1;
      const uint64_t drift = absd(diag(i) - diag(s));
      const int64_t gap = std::max(ts(i) - te(i - 1) - 1, qs(i) - qe(i - 1) - 1);
      if (drift > uint64_t(max_drift) || gap > max_drift || std::max(gt, gq) > max_win) break;
      if (gt >= 0 && gq >= 0) boundary = i;
    }
    bool adaptive;
    int64_t e;
    if (boundary >= 0) {
      adaptive = false;
      e = boundary;
    } else {
      e = s + 1;
      while (e < n && (ts(e) - te(s) - 1 < 0 || qs(e) - qe(s) - 1 < 0)) ++e;
      const uint64_t drift = absd(diag(e) - diag(s));
      const int64_t gap = std::max(ts(e) - te(s) - 1, qs(e) - qe(s) - 1);
      adaptive = drift > uint64_t(max_drift) || gap > max_drift;
    }
    if (e < n) {
      Anchor a = ch[size_t(e)];
      a.adaptive_before = adaptive;
      selected.push_back(a);
    } else {
      tail = adaptive;
    }
    s = e;
  }
  return {selected, tail};
}

// anchor_windows (src/minimizer.rs:466-479).
std::pair<std::vector<Anchor>, bool> anchor_windows(const HostParams &p, const uint8_t *q, int64_t qlen,
                                                    const uint8_t *consensus, int64_t clen) {
  const auto matches = collect_anchors(p, q, qlen, consensus, clen);
  const auto ch = chain(matches, int64_t(p.k));
  const int64_t max_win = std::min<int64_t>(int64_t(p.win_max), std::max<int64_t>(500, qlen / 25));
  return partition_windows(ch, clen, qlen, int64_t(p.win_band), max_win);
}

// src/minimizer.rs:505-578. Reads are compared by the minimizers they share:
// a minimizer value carried by more than mm_filter_ratio x n reads is
// dropped; per pair, the shared count is the sum over values of the smaller
// multiplicity, and the similarity is shared / (total_a + total_b - shared)
// weighted by 0.51 len_a / max_len + 0.49 len_b / max_len (so it is
// directional). The most similar ordered pair starts the order; each next
// read is the unused one of largest summed similarity to the reads already
// ordered (ties to the smaller index). Minimizers are this library's own
// (sketch above), so the order is the reference's only where the sketches
// agree.
std::vector<int64_t> guide_order(const HostParams &p, const std::vector<const uint8_t *> &seqs,
                                 const std::vector<int64_t> &lens) {
  const int64_t n = int64_t(seqs.size());
  std::vector<int64_t> input(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) input[size_t(i)] = i;
  if (!p.progressive || n < 2 || p.alphabet.size() > 5) return input;
  // value -> (read -> multiplicity), both in ascending order
  std::map<uint64_t, std::map<int64_t, int64_t>> groups;
  for (int64_t r = 0; r < n; ++r)
    for (const Minimizer &mm : sketch(seqs[size_t(r)], lens[size_t(r)], int64_t(p.k), int64_t(p.w)))
      ++groups[mm.value][r];
  if (groups.empty()) return input;
  std::vector<int64_t> total(static_cast<size_t>(n), 0), shared(static_cast<size_t>(n * n), 0);
  for (const auto &g : groups) {
    const auto &counts = g.second;
    if (double(counts.size()) > double(n) * p.mm_filter_ratio) continue;
    for (auto ia = counts.begin(); ia != counts.end(); ++ia) {
      const int64_t a = ia->first, ca = ia->second;
      total[size_t(a)] += ca;
      for (auto ib = counts.begin(); ib != ia; ++ib) {
        const int64_t b = ib->first, m = std::min(ca, ib->second);
        shared[size_t(a * n + b)] += m;
        shared[size_t(b * n + a)] += m;
      }
    }
  }
  int64_t mx = 1;
  for (int64_t l : lens) mx = std::max(mx, l);
  const double max_len = double(mx);
  std::vector<double> sim(static_cast<size_t>(n * n), 0.0);
  double best = -1.0;
  int64_t bi = 0, bj = 1;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j) {
      if (i == j) continue;
      const int64_t common = shared[size_t(i * n + j)];
      const int64_t uni = total[size_t(i)] + total[size_t(j)] - common;
      const double jac = uni == 0 ? 0.0
                                  : double(common) / double(uni) *
                                        (0.51 * double(lens[size_t(i)]) / max_len +
                                         0.49 * double(lens[size_t(j)]) / max_len);
      sim[size_t(i * n + j)] = jac;
      if (jac > best) {
        best = jac;
        bi = i;
        bj = j;
      }
    }
  std::vector<int64_t> order{bi, bj};
  std::vector<char> used(static_cast<size_t>(n), 0);
  used[size_t(bi)] = used[size_t(bj)] = 1;
  std::vector<double> sums(static_cast<size_t>(n));
  for (int64_t v = 0; v < n; ++v) sums[size_t(v)] = sim[size_t(bi * n + v)] + sim[size_t(bj * n + v)];
  while (int64_t(order.size()) < n) {
    int64_t next = -1;
    for (int64_t v = 0; v < n; ++v)
      if (!used[size_t(v)] && (next < 0 || sums[size_t(v)] > sums[size_t(next)])) next = v;
    order.push_back(next);
    used[size_t(next)] = 1;
    for (int64_t v = 0; v < n; ++v)
      if (!used[size_t(v)]) sums[size_t(v)] += sim[size_t(next * n + v)];
  }
  return order;
}

}  // namespace poa

// ---------------------------------------------------------------------------
// C ABI (host only; no CUDA context needed). Outputs are malloc'd and
// released with poa_free.

#include <cstdlib>
#include <cstring>

#include "../../include/minipoa_b200.h"

namespace {

using namespace poa;

template <class T>
int emit(const std::vector<T> &v, T **out, int64_t *n) {
  *out = static_cast<T *>(std::malloc(sizeof(T) * (v.size() + 1)));
  if (!*out) return POA_ERR_ALLOC;
  if (!v.empty()) std::memcpy(*out, v.data(), sizeof(T) * v.size());
  *n = int64_t(v.size());
  return POA_OK;
}

std::vector<poa_anchor> to_c(const std::vector<Anchor> &v) {
  std::vector<poa_anchor> o(v.size());
  for (size_t k = 0; k < v.size(); ++k)
    o[k] = poa_anchor{v[k].target_end, v[k].query_end, v[k].span, v[k].adaptive_before ? 1 : 0, 0};
  return o;
}

std::vector<Anchor> from_c(const poa_anchor *a, int64_t n) {
  std::vector<Anchor> o(size_t(std::max<int64_t>(n, 0)));
  for (int64_t k = 0; k < n; ++k) o[size_t(k)] = Anchor{a[k].target_end, a[k].query_end, a[k].span, a[k].adaptive_before != 0};
  return o;
}

bool valid_params(const poa_params *p, HostParams *hp) {
  if (!p) return false;
  *hp = HostParams::from(p);
  return hp->validate().empty();
}

}  // namespace

extern "C" {

int poa_seed_sketch(const uint8_t *seq, int64_t len, int64_t k, int64_t w, poa_minimizer **out, int64_t *n) {
  if (!out || !n || len < 0 || (len > 0 && !seq)) return POA_ERR_INVALID;
  std::vector<poa_minimizer> o;
  for (const Minimizer &m : sketch(seq, len, k, w)) o.push_back(poa_minimizer{m.value, m.end, m.span});
  return emit(o, out, n);
}

int poa_seed_repeat_intervals(const poa_minimizer *mm, int64_t n, int64_t len, int64_t max_dist, int64_t **out_pairs,
                              int64_t *n_out) {
  if (!out_pairs || !n_out || n < 0 || (n > 0 && !mm) || len < 0 || max_dist < 0) return POA_ERR_INVALID;
  std::vector<Minimizer> v;
  v.reserve(static_cast<size_t>(n));
  for (int64_t k = 0; k < n; ++k) v.push_back(Minimizer{mm[k].value, mm[k].end, mm[k].span});
  std::vector<int64_t> flat;
  for (auto &x : repeat_intervals(v, len, max_dist)) {
    flat.push_back(x.first);
    flat.push_back(x.second);
  }
  int64_t words = 0;
  const int rc = emit(flat, out_pairs, &words);
  *n_out = words / 2;
  return rc;
}

int poa_seed_collect_anchors(const poa_params *params, const uint8_t *q, int64_t qlen, const uint8_t *t, int64_t tlen,
                             poa_anchor **out, int64_t *n) {
  HostParams hp;
  if (!valid_params(params, &hp) || !out || !n || qlen < 0 || tlen < 0) return POA_ERR_INVALID;
  return emit(to_c(collect_anchors(hp, q, qlen, t, tlen)), out, n);
}

int poa_seed_chain(const poa_anchor *anchors, int64_t n, int64_t k, poa_anchor **out, int64_t *n_out) {
  if (!out || !n_out || n < 0 || (n > 0 && !anchors)) return POA_ERR_INVALID;
  return emit(to_c(chain(from_c(anchors, n), k)), out, n_out);
}

int poa_seed_partition_windows(const poa_anchor *ch, int64_t n, int64_t tlen, int64_t qlen, int64_t max_drift,
                               int64_t max_win, poa_anchor **out, int64_t *n_out, int32_t *tail_adaptive) {
  if (!out || !n_out || !tail_adaptive || n < 0 || (n > 0 && !ch)) return POA_ERR_INVALID;
  auto r = partition_windows(from_c(ch, n), tlen, qlen, max_drift, max_win);
  *tail_adaptive = r.second ? 1 : 0;
  return emit(to_c(r.first), out, n_out);
}

int poa_seed_anchor_windows(const poa_params *params, const uint8_t *q, int64_t qlen, const uint8_t *consensus,
                            int64_t clen, poa_anchor **out, int64_t *n_out, int32_t *tail_adaptive) {
  HostParams hp;
  if (!valid_params(params, &hp) || !out || !n_out || !tail_adaptive || qlen < 0 || clen < 0) return POA_ERR_INVALID;
  auto r = anchor_windows(hp, q, qlen, consensus, clen);
  *tail_adaptive = r.second ? 1 : 0;
  return emit(to_c(r.first), out, n_out);
}

int poa_seed_guide_order(const poa_params *params, int64_t n, const uint8_t *const *seqs, const int64_t *lens,
                         int64_t **out_order) {
  HostParams hp;
  if (!valid_params(params, &hp) || !out_order || n < 0 || (n > 0 && (!seqs || !lens))) return POA_ERR_INVALID;
  for (int64_t r = 0; r < n; ++r)
    if (lens[r] < 0 || (lens[r] > 0 && !seqs[r])) return POA_ERR_INVALID;
  int64_t n_out = 0;
  return emit(guide_order(hp, std::vector<const uint8_t *>(seqs, seqs + n), std::vector<int64_t>(lens, lens + n)),
              out_order, &n_out);
}

}  // extern "C"
