// Host side of the index: COO -> CSR grouping, the parallel block encoder
// (delta + bit-pack in blocks of 128 postings), the host decoder and the
// binary index file.
//
// The reference builds its mixed-container index single-threaded through a
// nested std::map (src/AdaBool/inverted_list.h:348-470) and re-parses text
// COO on every run (test/adsfilter_q_all.cu:127-161). Here the grouping is a
// counting sort, the encoder runs one contiguous term range per thread and
// concatenates, and the result can be stored as one binary file.
#include "abf_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <thread>
#include <mutex>

namespace abf {

int resolve_threads(int n) {
    if (n > 0) return n;
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? int(hc) : 1;
}

template <class F>
static void parallel_for(int n_threads, uint64_t n, F&& f) {
    n_threads = std::max(1, std::min<int>(n_threads, int(std::max<uint64_t>(n, 1))));
    if (n_threads == 1) {
        f(0, 0, n);
        return;
    }
    std::vector<std::thread> th;
    uint64_t per = (n + n_threads - 1) / n_threads;
    for (int i = 0; i < n_threads; ++i) {
        uint64_t b = std::min<uint64_t>(n, per * i), e = std::min<uint64_t>(n, b + per);
        th.emplace_back([&, i, b, e] { f(i, b, e); });
    }
    for (auto& t : th) t.join();
}

abf_status coo_to_csr(const uint32_t* terms, const uint32_t* ads, uint64_t nnz, uint32_t n_terms,
                      uint32_t n_ads, int n_threads, std::vector<uint64_t>* offsets,
                      std::vector<uint32_t>* csr_ads) {
    n_threads = std::min(resolve_threads(n_threads), 16);
    std::vector<std::vector<uint64_t>> hist(n_threads);
    std::atomic<bool> bad{false};
    uint64_t per = (nnz + n_threads - 1) / std::max(n_threads, 1);
    std::vector<std::thread> th;
    for (int i = 0; i < n_threads; ++i) {
        th.emplace_back([&, i] {
            auto& h = hist[i];
            h.assign(size_t(n_terms) + 1, 0);
            uint64_t b = std::min(nnz, per * i), e = std::min(nnz, b + per);
            for (uint64_t k = b; k < e; ++k) {
                if (terms[k] >= n_terms || ads[k] >= n_ads) {
                    bad = true;
                    return;
                }
                ++h[terms[k]];
            }
        });
    }
    for (auto& t : th) t.join();
    if (bad) return fail(ABF_ERR_RANGE, "COO pair outside [0,n_terms) x [0,n_ads)");
    offsets->assign(size_t(n_terms) + 1, 0);
    // per-thread write cursors: term-major, thread-minor, so each term's ads
    // keep their input order (not needed for correctness, sorting follows)
    uint64_t run = 0;
    for (uint32_t t = 0; t < n_terms; ++t) {
        (*offsets)[t] = run;
        for (int i = 0; i < n_threads; ++i) {
            uint64_t c = hist[i][t];
            hist[i][t] = run;
            run += c;
        }
    }
    (*offsets)[n_terms] = run;
    csr_ads->resize(nnz);
    th.clear();
    for (int i = 0; i < n_threads; ++i) {
        th.emplace_back([&, i] {
            auto& h = hist[i];
            uint64_t b = std::min(nnz, per * i), e = std::min(nnz, b + per);
            for (uint64_t k = b; k < e; ++k) (*csr_ads)[h[terms[k]]++] = ads[k];
        });
    }
    for (auto& t : th) t.join();
    return ABF_OK;
}

namespace {

struct Chunk {
    uint32_t t0 = 0, t1 = 0;
    std::vector<uint32_t> nblk, len;  // per term of the chunk
    std::vector<uint32_t> first, last;
    std::vector<abf_u2> desc;
    std::vector<uint32_t> words;      // payload as uint32 words (multiple of 4)
    uint32_t max_len = 0;
    uint64_t postings = 0;
    bool bad = false;
};

inline uint32_t bit_width(uint32_t v) { return v ? 32u - uint32_t(__builtin_clz(v)) : 0u; }

void encode_list(const uint32_t* ids, uint32_t n, Chunk& c) {
    for (uint32_t i0 = 0; i0 < n; i0 += kBlock) {
        uint32_t cnt = std::min(kBlock, n - i0);
        const uint32_t* x = ids + i0;
        uint32_t maxv = 0;
        for (uint32_t s = 0; s + 1 < cnt; ++s) maxv = std::max(maxv, x[s + 1] - x[s] - 1u);
        uint32_t bits = bit_width(maxv);
        uint32_t units = payload_units(cnt, bits);
        size_t w0 = c.words.size();
        c.first.push_back(x[0]);
        c.last.push_back(x[cnt - 1]);
        c.desc.push_back(abf_u2{uint32_t(w0 / 4), make_meta(bits, cnt)});
        c.words.resize(w0 + size_t(units) * 4, 0u);
        if (bits == 0) continue;
        uint32_t* w = c.words.data() + w0;
        for (uint32_t s = 0; s + 1 < cnt; ++s) {
            uint32_t v = x[s + 1] - x[s] - 1u;
            uint64_t pos = uint64_t(s) * bits;
            uint32_t wi = uint32_t(pos >> 5), sh = uint32_t(pos & 31);
            w[wi] |= v << sh;
            if (sh + bits > 32) w[wi + 1] |= v >> (32 - sh);
        }
    }
}

}  // namespace

abf_status build_host(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, uint32_t n_ads,
                      int n_threads, HostIndex* out) {
    n_threads = resolve_threads(n_threads);
    uint64_t nnz = offsets[n_terms];
    // split terms into ~equal-posting chunks, a few per thread
    int n_chunks = std::max(1, std::min<int>(n_threads * 4, int(std::max<uint32_t>(n_terms, 1))));
    std::vector<Chunk> chunks(n_chunks);
    {
        uint32_t t = 0;
        for (int i = 0; i < n_chunks; ++i) {
            uint64_t goal = (nnz * uint64_t(i + 1)) / uint64_t(n_chunks);
            uint32_t t0 = t;
            if (i == n_chunks - 1) {
                t = n_terms;
            } else {
                // first term whose end offset exceeds goal
                uint32_t lo = t, hi = n_terms;
                while (lo < hi) {
                    uint32_t mid = lo + (hi - lo) / 2;
                    if (offsets[mid + 1] <= goal) lo = mid + 1; else hi = mid;
                }
                t = std::max(t, lo);
            }
            chunks[i].t0 = t0;
            chunks[i].t1 = t;
        }
    }
    std::atomic<int> next{0};
    auto worker = [&](int, uint64_t, uint64_t) {
        std::vector<uint32_t> tmp;
        for (;;) {
            int ci = next.fetch_add(1);
            if (ci >= n_chunks) break;
            Chunk& c = chunks[ci];
            c.nblk.reserve(c.t1 - c.t0);
            c.len.reserve(c.t1 - c.t0);
            for (uint32_t t = c.t0; t < c.t1; ++t) {
                uint64_t b = offsets[t], e = offsets[t + 1];
                const uint32_t* ids = ads + b;
                uint64_t n = e - b;
                bool ok = true;
                for (uint64_t k = 0; k < n; ++k) {
                    if (ids[k] >= n_ads) { c.bad = true; break; }
                    if (k && ids[k] <= ids[k - 1]) ok = false;
                }
                if (c.bad) return;
                if (!ok) {  // unsorted or duplicated: sort and merge a copy
                    tmp.assign(ids, ids + n);
                    std::sort(tmp.begin(), tmp.end());
                    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
                    ids = tmp.data();
                    n = tmp.size();
                }
                size_t nb0 = c.first.size();
                encode_list(ids, uint32_t(n), c);
                c.nblk.push_back(uint32_t(c.first.size() - nb0));
                c.len.push_back(uint32_t(n));
                c.max_len = std::max<uint32_t>(c.max_len, uint32_t(n));
                c.postings += n;
            }
        }
    };
    parallel_for(n_threads, uint64_t(n_threads), worker);
    for (auto& c : chunks)
        if (c.bad) return fail(ABF_ERR_RANGE, "ad id >= n_ads in a posting list");

    // concatenate
    std::vector<uint64_t> blk_base(n_chunks + 1, 0), unit_base(n_chunks + 1, 0);
    for (int i = 0; i < n_chunks; ++i) {
        blk_base[i + 1] = blk_base[i] + chunks[i].first.size();
        unit_base[i + 1] = unit_base[i] + chunks[i].words.size() / 4;
    }
    uint64_t n_blocks = blk_base[n_chunks], n_units = unit_base[n_chunks];
    if (n_blocks >= (1ull << 32) || n_units >= (1ull << 32))
        return fail(ABF_ERR_RANGE, "index too large for 32-bit block/payload offsets");
    out->n_terms = n_terms;
    out->n_ads = n_ads;
    out->term_blk.assign(size_t(n_terms) + 1, 0);
    out->term_len.assign(n_terms, 0);
    out->blk_first.resize(n_blocks);
    out->blk_last.resize(n_blocks);
    out->blk_term.resize(n_blocks);
    out->blk_desc.resize(n_blocks);
    out->payload.assign(n_units + 1, abf_u4{0, 0, 0, 0});
    out->n_postings = 0;
    out->max_list_len = 0;
    for (auto& c : chunks) {
        out->n_postings += c.postings;
        out->max_list_len = std::max(out->max_list_len, c.max_len);
    }
    parallel_for(n_threads, uint64_t(n_chunks), [&](int, uint64_t cb, uint64_t ce) {
        for (uint64_t ci = cb; ci < ce; ++ci) {
            Chunk& c = chunks[ci];
            uint64_t bb = blk_base[ci];
            uint32_t run = uint32_t(bb);
            for (uint32_t t = c.t0; t < c.t1; ++t) {
                uint32_t k = t - c.t0;
                out->term_blk[t] = run;
                out->term_len[t] = c.len[k];
                for (uint32_t j = 0; j < c.nblk[k]; ++j) out->blk_term[run + j] = t;
                run += c.nblk[k];
            }
            std::copy(c.first.begin(), c.first.end(), out->blk_first.begin() + bb);
            std::copy(c.last.begin(), c.last.end(), out->blk_last.begin() + bb);
            for (size_t j = 0; j < c.desc.size(); ++j) {
                abf_u2 d = c.desc[j];
                d.x += uint32_t(unit_base[ci]);
                out->blk_desc[bb + j] = d;
            }
            if (!c.words.empty())
                std::memcpy(reinterpret_cast<uint32_t*>(out->payload.data()) + unit_base[ci] * 4,
                            c.words.data(), c.words.size() * 4);
            std::vector<uint32_t>().swap(c.words);
        }
    });
    out->term_blk[n_terms] = uint32_t(n_blocks);
    return ABF_OK;
}

void decode_block_host(const HostIndex& h, uint64_t b, uint32_t* out) {
    abf_u2 d = h.blk_desc[b];
    uint32_t bits = desc_bits(d.y), cnt = desc_count(d.y);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(h.payload.data()) + size_t(d.x) * 4;
    uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
    uint32_t id = h.blk_first[b];
    out[0] = id;
    for (uint32_t s = 0; s + 1 < cnt; ++s) {
        uint32_t v = 0;
        if (bits) {
            uint64_t pos = uint64_t(s) * bits;
            uint32_t wi = uint32_t(pos >> 5), sh = uint32_t(pos & 31);
            uint64_t win = uint64_t(w[wi]) | (sh + bits > 32 ? uint64_t(w[wi + 1]) << 32 : 0);
            v = uint32_t(win >> sh) & mask;
        }
        id += v + 1u;
        out[s + 1] = id;
    }
}

void derive_tables(const HostIndex& h, uint32_t dense_div, int n_threads, DerivedHost* out) {
    n_threads = resolve_threads(n_threads);
    const uint64_t n_words = (uint64_t(h.n_ads) + 31) / 32;
    out->dense_stride = (n_words + 3) & ~uint64_t(3);
    out->term_dense.assign(h.n_terms, kNone);
    out->term_dir.assign(h.n_terms, kNone);
    out->dir_n = uint32_t(((uint64_t(h.n_ads) + (1u << kDirShift) - 1) >> kDirShift) + 1);
    if (dense_div == 0) dense_div = kDefaultDenseDiv;
    // dense candidates, longest first, within a memory budget of twice the
    // payload (at least 256 MB)
    std::vector<uint32_t> cand;
    for (uint32_t t = 0; t < h.n_terms; ++t)
        if (dense_div != kNone && h.term_len[t] && uint64_t(h.term_len[t]) * dense_div >= h.n_ads) cand.push_back(t);
    std::sort(cand.begin(), cand.end(), [&](uint32_t a, uint32_t b) { return h.term_len[a] > h.term_len[b]; });
    const uint64_t budget = std::max<uint64_t>(256ull << 20, 2ull * 16ull * h.payload.size());
    std::vector<uint32_t> dense_terms;
    for (uint32_t t : cand) {
        // 16-bit bitmap indices in the merge kernels' per-query lists
        if ((dense_terms.size() + 1) * out->dense_stride * 4 > budget || dense_terms.size() >= 65535) break;
        out->term_dense[t] = uint32_t(dense_terms.size());
        dense_terms.push_back(t);
    }
    out->n_dense = uint32_t(dense_terms.size());
    std::vector<uint32_t> dir_terms;
    for (uint32_t t = 0; t < h.n_terms; ++t) {
        if (out->term_dense[t] != kNone) continue;
        if (uint64_t(h.term_len[t]) * kDirDiv >= h.n_ads && h.term_blk[t + 1] - h.term_blk[t] >= 2) {
            out->term_dir[t] = uint32_t(dir_terms.size()) * out->dir_n;
            dir_terms.push_back(t);
        }
    }
    out->n_dir = uint32_t(dir_terms.size());
    out->dense.assign(size_t(out->n_dense) * out->dense_stride, 0u);
    out->dir.assign(size_t(out->n_dir) * out->dir_n, 0u);
    parallel_for(n_threads, out->n_dense, [&](int, uint64_t b, uint64_t e) {
        uint32_t buf[kBlock];
        for (uint64_t i = b; i < e; ++i) {
            const uint32_t t = dense_terms[i];
            uint32_t* bm = out->dense.data() + i * out->dense_stride;
            for (uint32_t blk = h.term_blk[t]; blk < h.term_blk[t + 1]; ++blk) {
                decode_block_host(h, blk, buf);
                const uint32_t cnt = desc_count(h.blk_desc[blk].y);
                for (uint32_t k = 0; k < cnt; ++k) bm[buf[k] >> 5] |= 1u << (buf[k] & 31u);
            }
        }
    });
    parallel_for(n_threads, out->n_dir, [&](int, uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const uint32_t t = dir_terms[i];
            uint32_t* d = out->dir.data() + i * out->dir_n;
            uint32_t blk = h.term_blk[t];
            const uint32_t b1 = h.term_blk[t + 1];
            for (uint32_t j = 0; j < out->dir_n; ++j) {
                const uint64_t lo = uint64_t(j) << kDirShift;
                while (blk < b1 && uint64_t(h.blk_last[blk]) < lo) ++blk;
                d[j] = blk;
            }
        }
    });
}

}  // namespace abf

// ---------------------------------------------------------------------------
// binary index file
// ---------------------------------------------------------------------------
namespace {
const char kMagic[8] = {'A', 'B', 'F', 'I', 'D', 'X', '0', '1'};
struct FileHeader {
    char magic[8];
    uint32_t version, block;
    uint32_t n_terms, n_ads;
    uint64_t n_postings, n_blocks, n_units;
    uint32_t max_list_len, pad;
};

template <class T>
bool write_vec(std::FILE* f, const std::vector<T>& v) {
    return v.empty() || std::fwrite(v.data(), sizeof(T), v.size(), f) == v.size();
}
template <class T>
bool read_vec(std::FILE* f, std::vector<T>& v, uint64_t n) {
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}
}  // namespace

namespace abf {
abf_status save_host(const HostIndex& h, const char* path) {
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return fail(ABF_ERR_IO, std::string("cannot open for writing: ") + path);
    FileHeader hd{};
    std::memcpy(hd.magic, kMagic, 8);
    hd.version = ABF_ABI_VERSION;
    hd.block = kBlock;
    hd.n_terms = h.n_terms;
    hd.n_ads = h.n_ads;
    hd.n_postings = h.n_postings;
    hd.n_blocks = h.n_blocks();
    hd.n_units = h.payload.size();
    hd.max_list_len = h.max_list_len;
    bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 && write_vec(f, h.term_blk) &&
              write_vec(f, h.term_len) && write_vec(f, h.blk_first) && write_vec(f, h.blk_last) &&
              write_vec(f, h.blk_term) && write_vec(f, h.blk_desc) && write_vec(f, h.payload);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? ABF_OK : fail(ABF_ERR_IO, std::string("write failed: ") + path);
}

abf_status load_host(const char* path, HostIndex* h) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ABF_ERR_IO, std::string("cannot open: ") + path);
    FileHeader hd{};
    bool ok = std::fread(&hd, sizeof(hd), 1, f) == 1 && std::memcmp(hd.magic, kMagic, 8) == 0 &&
              hd.block == kBlock && hd.n_blocks < (1ull << 32) && hd.n_units < (1ull << 33);
    if (ok) {
        h->n_terms = hd.n_terms;
        h->n_ads = hd.n_ads;
        h->n_postings = hd.n_postings;
        h->max_list_len = hd.max_list_len;
        ok = read_vec(f, h->term_blk, uint64_t(hd.n_terms) + 1) && read_vec(f, h->term_len, hd.n_terms) &&
             read_vec(f, h->blk_first, hd.n_blocks) && read_vec(f, h->blk_last, hd.n_blocks) &&
             read_vec(f, h->blk_term, hd.n_blocks) && read_vec(f, h->blk_desc, hd.n_blocks) &&
             read_vec(f, h->payload, hd.n_units);
    }
    std::fclose(f);
    if (!ok) return fail(ABF_ERR_IO, std::string("not an index file or truncated: ") + path);
    // structural checks so a corrupt file cannot send a kernel out of bounds
    if (h->term_blk[0] != 0 || h->term_blk[h->n_terms] != hd.n_blocks || h->payload.empty())
        return fail(ABF_ERR_IO, "index file: inconsistent block table");
    for (uint32_t t = 0; t < h->n_terms; ++t)
        if (h->term_blk[t + 1] < h->term_blk[t]) return fail(ABF_ERR_IO, "index file: term table not monotone");
    for (uint64_t b = 0; b < hd.n_blocks; ++b) {
        abf_u2 d = h->blk_desc[b];
        uint32_t bits = desc_bits(d.y), cnt = desc_count(d.y);
        if (bits > 32 || cnt > kBlock || uint64_t(d.x) + payload_units(cnt, bits) > hd.n_units ||
            h->blk_first[b] >= h->n_ads || h->blk_last[b] >= h->n_ads || h->blk_term[b] >= h->n_terms)
            return fail(ABF_ERR_IO, "index file: bad block descriptor");
    }
    return ABF_OK;
}
}  // namespace abf
