// Seeded synthetic filter matrices and query sets (include/abf_workload.h).
//
// Random numbers: SplitMix64 (Steele, Lea, Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014), one independent stream per
// term or per query, keyed by (seed, id), so results do not depend on how
// the work is split across threads.
#include "abf_internal.h"
#include "../../include/abf_workload.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed, uint64_t stream) {
        s = seed * 0x9E3779B97F4A7C15ull ^ (stream + 0x632BE59BD9B4E019ull) * 0xD1B54A32D192ED03ull;
        next();
    }
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // uniform in (0, 1]
    double unit() { return double((next() >> 11) + 1) * (1.0 / 9007199254740992.0); }
};

template <class F>
void dynamic_for(int n_threads, uint64_t n, uint64_t grain, F&& f) {
    n_threads = abf::resolve_threads(n_threads);
    std::atomic<uint64_t> next{0};
    auto body = [&] {
        for (;;) {
            uint64_t b = next.fetch_add(grain);
            if (b >= n) break;
            uint64_t e = std::min(n, b + grain);
            for (uint64_t i = b; i < e; ++i) f(i);
        }
    };
    if (n_threads <= 1 || n <= grain) {
        body();
        return;
    }
    std::vector<std::thread> th;
    for (int i = 0; i < n_threads; ++i) th.emplace_back(body);
    for (auto& t : th) t.join();
}

bool valid(const abf_gen_lists_params* p) {
    return p && p->n_terms > 0 && p->n_ads > 0 && p->zipf_s > 0 && p->max_len > 0;
}

// Bernoulli(len / n_ads) selection of ads for one term; calls emit(ad) in
// ascending order, returns the count. At least one ad is selected.
template <class Emit>
uint64_t draw_list(uint64_t seed, uint32_t term, uint32_t len, uint32_t n_ads, Emit&& emit) {
    Rng r(seed ^ 0x5bd1e995ull, term);
    uint64_t cnt = 0;
    if (len >= n_ads) {
        for (uint32_t a = 0; a < n_ads; ++a) emit(a);
        return n_ads;
    }
    double p = double(len) / double(n_ads);
    if (p >= 1.0 / 16.0) {
        uint64_t thr = uint64_t(p * 4294967296.0);
        for (uint32_t a = 0; a < n_ads; ++a) {
            if ((r.next() >> 32) < thr) {
                emit(a);
                ++cnt;
            }
        }
    } else {
        double inv = 1.0 / std::log1p(-p);
        int64_t a = -1;
        for (;;) {
            double g = std::floor(std::log(r.unit()) * inv);
            if (g >= double(n_ads)) break;
            a += int64_t(g) + 1;
            if (a >= int64_t(n_ads)) break;
            emit(uint32_t(a));
            ++cnt;
        }
    }
    if (cnt == 0) {
        emit(uint32_t(r.next() % n_ads));
        cnt = 1;
    }
    return cnt;
}

}  // namespace

extern "C" abf_status abf_gen_target_lengths(const abf_gen_lists_params* p, uint32_t* out) {
    if (!valid(p) || !out) return abf::fail(ABF_ERR_INVALID, "abf_gen_target_lengths: bad parameters");
    uint32_t n = p->n_terms;
    std::vector<double> f(n);
    for (uint32_t r = 0; r < n; ++r) f[r] = std::pow(double(r + 1), -p->zipf_s);
    auto total = [&](double c) {
        double s = 0;
        for (uint32_t r = 0; r < n; ++r) s += std::min(double(p->max_len), std::max(1.0, std::round(c * f[r])));
        return s;
    };
    double target = double(p->nnz_target);
    double lo = 0, hi = 1;
    while (total(hi) < target && hi < 1e300) hi *= 2;
    for (int it = 0; it < 100; ++it) {
        double mid = 0.5 * (lo + hi);
        (total(mid) < target ? lo : hi) = mid;
    }
    double c = hi;
    // rank -> term permutation (Fisher-Yates)
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    Rng r(p->seed, 0xABCDEF12ull);
    for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[uint32_t(r.next() % (uint64_t(i) + 1))]);
    uint32_t cap = std::min(p->max_len, p->n_ads);
    for (uint32_t rk = 0; rk < n; ++rk) {
        double v = std::min(double(cap), std::max(1.0, std::round(c * f[rk])));
        out[perm[rk]] = uint32_t(v);
    }
    return ABF_OK;
}

extern "C" abf_status abf_gen_lists_offsets(const abf_gen_lists_params* p, uint64_t* off) {
    if (!valid(p) || !off) return abf::fail(ABF_ERR_INVALID, "abf_gen_lists_offsets: bad parameters");
    std::vector<uint32_t> len(p->n_terms);
    abf_status st = abf_gen_target_lengths(p, len.data());
    if (st != ABF_OK) return st;
    std::vector<uint64_t> cnt(p->n_terms);
    dynamic_for(p->n_threads, p->n_terms, 64, [&](uint64_t t) {
        cnt[t] = draw_list(p->seed, uint32_t(t), len[t], p->n_ads, [](uint32_t) {});
    });
    off[0] = 0;
    for (uint32_t t = 0; t < p->n_terms; ++t) off[t + 1] = off[t] + cnt[t];
    return ABF_OK;
}

extern "C" abf_status abf_gen_lists_fill(const abf_gen_lists_params* p, const uint64_t* off, uint32_t* ads) {
    if (!valid(p) || !off || !ads) return abf::fail(ABF_ERR_INVALID, "abf_gen_lists_fill: bad parameters");
    std::vector<uint32_t> len(p->n_terms);
    abf_status st = abf_gen_target_lengths(p, len.data());
    if (st != ABF_OK) return st;
    std::atomic<bool> mismatch{false};
    dynamic_for(p->n_threads, p->n_terms, 64, [&](uint64_t t) {
        uint32_t* dst = ads + off[t];
        uint64_t k = 0, cap = off[t + 1] - off[t];
        uint64_t n = draw_list(p->seed, uint32_t(t), len[t], p->n_ads, [&](uint32_t a) {
            if (k < cap) dst[k] = a;
            ++k;
        });
        if (n != cap) mismatch = true;
    });
    if (mismatch) return abf::fail(ABF_ERR_INVALID, "abf_gen_lists_fill: offsets do not match these parameters");
    return ABF_OK;
}

namespace {
uint32_t query_count(const abf_gen_queries_params* p, uint32_t q, uint32_t nonempty) {
    Rng r(p->seed ^ 0x1234567ull, q);
    uint64_t c;
    if (p->count_kind == ABF_QCOUNT_UNIFORM) {
        c = p->lo + r.next() % (uint64_t(p->hi) - p->lo + 1);
    } else {
        double u1 = r.unit(), u2 = r.unit();
        double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
        double v = std::round(p->median * std::exp(p->sigma * z));
        v = std::min(double(p->hi), std::max(double(p->lo), v));
        c = uint64_t(v);
    }
    return uint32_t(std::min<uint64_t>(c, nonempty));
}
}  // namespace

extern "C" abf_status abf_gen_queries_offsets(const abf_gen_queries_params* p, const uint32_t* len,
                                              uint32_t n_terms, uint64_t* off) {
    if (!p || !len || !off || p->lo > p->hi || n_terms == 0)
        return abf::fail(ABF_ERR_INVALID, "abf_gen_queries_offsets: bad parameters");
    uint32_t nonempty = 0;
    for (uint32_t t = 0; t < n_terms; ++t) nonempty += len[t] > 0;
    off[0] = 0;
    for (uint32_t q = 0; q < p->n_queries; ++q) off[q + 1] = off[q] + query_count(p, q, nonempty);
    return ABF_OK;
}

extern "C" abf_status abf_gen_queries_fill(const abf_gen_queries_params* p, const uint32_t* len, uint32_t n_terms,
                                           const uint64_t* off, uint32_t* out) {
    if (!p || !len || !off || !out || n_terms == 0)
        return abf::fail(ABF_ERR_INVALID, "abf_gen_queries_fill: bad parameters");
    std::vector<uint64_t> cum(size_t(n_terms) + 1, 0);
    for (uint32_t t = 0; t < n_terms; ++t) cum[t + 1] = cum[t] + len[t];
    uint64_t total = cum[n_terms];
    if (total == 0) return abf::fail(ABF_ERR_INVALID, "abf_gen_queries_fill: all lists empty");
    dynamic_for(p->n_threads, p->n_queries, 16, [&](uint64_t q) {
        uint32_t k = uint32_t(off[q + 1] - off[q]);
        uint32_t* dst = out + off[q];
        Rng r(p->seed ^ 0x9876543ull, q);
        // open-addressing set of chosen terms
        uint32_t cap = 16;
        while (cap < 2 * k + 2) cap <<= 1;
        std::vector<uint32_t> set(cap, 0xffffffffu);
        auto insert = [&](uint32_t t) {
            uint32_t h = (t * 2654435761u) & (cap - 1);
            while (set[h] != 0xffffffffu) {
                if (set[h] == t) return false;
                h = (h + 1) & (cap - 1);
            }
            set[h] = t;
            return true;
        };
        uint32_t got = 0;
        uint64_t tries = 0, max_tries = 64ull * k + 1024;
        while (got < k && tries < max_tries) {
            ++tries;
            uint64_t x = r.next() % total;
            uint32_t t = uint32_t(std::upper_bound(cum.begin(), cum.end(), x) - cum.begin()) - 1;
            if (insert(t)) dst[got++] = t;
        }
        if (got < k) {
            // heavily skewed tiny index: finish with the unchosen non-empty
            // terms in a seeded random order
            std::vector<uint32_t> rest;
            for (uint32_t t = 0; t < n_terms; ++t) {
                if (!len[t]) continue;
                uint32_t h = (t * 2654435761u) & (cap - 1);
                bool seen = false;
                while (set[h] != 0xffffffffu) {
                    if (set[h] == t) { seen = true; break; }
                    h = (h + 1) & (cap - 1);
                }
                if (!seen) rest.push_back(t);
            }
            for (size_t i = rest.size(); i > 1; --i) std::swap(rest[i - 1], rest[r.next() % i]);
            for (size_t i = 0; got < k && i < rest.size(); ++i) dst[got++] = rest[i];
        }
    });
    return ABF_OK;
}
