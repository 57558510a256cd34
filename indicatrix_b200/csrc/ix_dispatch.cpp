// ix_dispatch.cpp -- SampleCursor and Merger (include/ix_dispatch.h).
//
// Semantics follow crates/indicatrix-dispatch/src/sample_cursor/mod.rs:64-230 and
// merge/mod.rs:155-460: ranges are claimed in ascending order (re-queued ranges first);
// the merge is a left fold in ascending first-sample order starting from zero, so for a
// given partition into chunks the merged sums are bit-identical whichever lane traced
// which chunk and whenever it finished.

#include "../../include/ix_dispatch.h"

#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <vector>

struct ix_sample_cursor {
    std::mutex mu;
    uint32_t next, end;
    std::deque<std::pair<uint32_t, uint32_t>> requeued;
};

// A byte budget several mergers park against (ParkedBudget, merge/mod.rs:72-80): reserve
// refuses past the cap, release returns bytes; thread-safe.
struct ix_parked_budget {
    std::mutex mu;
    uint64_t cap, used = 0;
    bool reserve(uint64_t bytes) {
        std::lock_guard<std::mutex> lk(mu);
        if (used + bytes > cap) return false;
        used += bytes;
        return true;
    }
    void release(uint64_t bytes) {
        std::lock_guard<std::mutex> lk(mu);
        used -= bytes < used ? bytes : used;
    }
};

struct ix_merger {
    struct Parked {
        uint32_t done;
        std::vector<double> sum;
    };
    mutable std::mutex mu;
    uint64_t pixels;
    uint32_t first_sample;
    // The budget parked chunks are charged against: the merger's own (ix_merger_new with a
    // nonzero size), a shared one (ix_merger_new_shared), or none.
    ix_parked_budget* budget = nullptr;
    bool owns_budget = false;
    std::vector<double> merged;
    uint32_t merged_count = 0, parked_count = 0;
    uint32_t frontier;
    std::map<uint32_t, Parked> parked;
    uint64_t dropped_pixels = 0;
};

namespace {

void add_assign(std::vector<double>& dst, const std::vector<double>& src) {
    if (dst.empty()) dst.assign(src.size(), 0.0);
    for (size_t i = 0; i < src.size(); ++i) dst[i] += src[i];
}

// Merger::add's overlap test (merge/mod.rs overlaps()).
bool overlaps(const ix_merger& m, uint32_t first, uint32_t done) {
    const uint64_t end = (uint64_t)first + done;
    if (first < m.frontier) return true;
    auto after = m.parked.lower_bound(first);
    if (after != m.parked.begin()) {
        auto before = std::prev(after);
        if ((uint64_t)before->first + before->second.done > first) return true;
    }
    if (after != m.parked.end() && after->first < end) return true;
    return false;
}

void advance_frontier(ix_merger& m) {
    for (;;) {
        auto it = m.parked.find(m.frontier);
        if (it == m.parked.end()) break;
        add_assign(m.merged, it->second.sum);
        m.frontier += it->second.done;
        m.merged_count += it->second.done;
        m.parked_count -= it->second.done;
        m.parked.erase(it);
    }
}

}  // namespace

extern "C" {

ix_sample_cursor* ix_sample_cursor_new(uint32_t start, uint32_t end) {
    ix_sample_cursor* c = new ix_sample_cursor();
    c->next = start;
    c->end = end;
    return c;
}

void ix_sample_cursor_free(ix_sample_cursor* c) { delete c; }

int ix_sample_cursor_claim(ix_sample_cursor* c, uint32_t want, uint32_t* start, uint32_t* count) {
    if (!c || want == 0) return 0;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->requeued.empty()) {
        auto r = c->requeued.front();
        uint32_t take = want < r.second ? want : r.second;
        *start = r.first;
        *count = take;
        if (take == r.second)
            c->requeued.pop_front();
        else
            c->requeued.front() = {r.first + take, r.second - take};
        return 1;
    }
    if (c->next >= c->end) return 0;
    uint32_t s = c->next;
    uint64_t e = (uint64_t)s + want;
    c->next = (uint32_t)(e < c->end ? e : c->end);
    *start = s;
    *count = c->next - s;
    return 1;
}

void ix_sample_cursor_requeue(ix_sample_cursor* c, uint32_t start, uint32_t count) {
    if (!c || count == 0) return;
    std::lock_guard<std::mutex> lk(c->mu);
    c->requeued.emplace_back(start, count);
}

int ix_sample_cursor_fully_claimed(const ix_sample_cursor* c) {
    if (!c) return 1;
    std::lock_guard<std::mutex> lk(const_cast<ix_sample_cursor*>(c)->mu);
    return (c->next >= c->end && c->requeued.empty()) ? 1 : 0;
}

ix_parked_budget* ix_parked_budget_new(uint64_t bytes) {
    ix_parked_budget* b = new ix_parked_budget();
    b->cap = bytes;
    return b;
}

void ix_parked_budget_free(ix_parked_budget* b) { delete b; }

uint64_t ix_parked_budget_used(ix_parked_budget* b) {
    if (!b) return 0;
    std::lock_guard<std::mutex> lk(b->mu);
    return b->used;
}

ix_merger* ix_merger_new(uint64_t pixels, uint32_t first_sample, uint64_t parked_budget_bytes) {
    ix_merger* m = new ix_merger();
    m->pixels = pixels;
    m->first_sample = first_sample;
    m->frontier = first_sample;
    if (parked_budget_bytes) {
        m->budget = ix_parked_budget_new(parked_budget_bytes);
        m->owns_budget = true;
    }
    return m;
}

ix_merger* ix_merger_new_shared(uint64_t pixels, uint32_t first_sample, ix_parked_budget* budget) {
    ix_merger* m = ix_merger_new(pixels, first_sample, 0);
    m->budget = budget;
    return m;
}

void ix_merger_free(ix_merger* m) {
    if (!m) return;
    // A merger dropped with chunks still parked returns their charge (merge/tests.rs:172).
    if (m->budget && !m->parked.empty()) m->budget->release(m->parked.size() * m->pixels * 3 * sizeof(double));
    if (m->owns_budget) delete m->budget;
    delete m;
}

int ix_merger_add(ix_merger* m, uint32_t first_sample, uint32_t done, const double* sums, uint64_t len,
                  uint32_t* total) {
    if (!m) return IX_MERGE_WRONG_LENGTH;
    if (done == 0) {
        if (total) *total = ix_merger_total(m);
        return IX_MERGE_OK;
    }
    if (len != m->pixels * 3 || !sums) return IX_MERGE_WRONG_LENGTH;
    // zero_invalid_pixels: a pixel with a non-finite or negative component is dropped.
    std::vector<double> sum(sums, sums + len);
    uint64_t dropped = 0;
    for (uint64_t p = 0; p < m->pixels; ++p) {
        double* v = sum.data() + 3 * p;
        bool ok = true;
        for (int k = 0; k < 3; ++k) ok = ok && std::isfinite(v[k]) && v[k] >= 0.0;
        if (!ok) {
            v[0] = v[1] = v[2] = 0.0;
            ++dropped;
        }
    }
    std::lock_guard<std::mutex> lk(m->mu);
    if (overlaps(*m, first_sample, done)) return IX_MERGE_OVERLAP;
    const size_t before = m->parked.size();
    m->parked[first_sample] = ix_merger::Parked{done, std::move(sum)};
    m->parked_count += done;
    advance_frontier(*m);
    const size_t after = m->parked.size();
    const uint64_t chunk_bytes = m->pixels * 3 * sizeof(double);
    if (m->budget) {
        // Only a chunk that stays parked needs budget; folded chunks release theirs.
        if (after > before) {
            if (!m->budget->reserve(chunk_bytes)) {
                m->parked.erase(first_sample);
                m->parked_count -= done;
                return IX_MERGE_BUDGET;
            }
        } else if (after < before) {
            m->budget->release(chunk_bytes * (before - after));
        }
    }
    m->dropped_pixels += dropped;
    if (total) *total = m->merged_count + m->parked_count;
    return IX_MERGE_OK;
}

uint32_t ix_merger_frontier(const ix_merger* m) {
    std::lock_guard<std::mutex> lk(m->mu);
    return m->frontier;
}

uint32_t ix_merger_total(const ix_merger* m) {
    std::lock_guard<std::mutex> lk(m->mu);
    return m->merged_count + m->parked_count;
}

uint64_t ix_merger_dropped_pixels(const ix_merger* m) {
    std::lock_guard<std::mutex> lk(m->mu);
    return m->dropped_pixels;
}

uint32_t ix_merger_snapshot(const ix_merger* m, double* dst, uint64_t len) {
    if (!m || !dst || len != m->pixels * 3) return 0;
    std::lock_guard<std::mutex> lk(m->mu);
    for (size_t i = 0; i < m->merged.size(); ++i) dst[i] += m->merged[i];
    for (const auto& kv : m->parked)
        for (size_t i = 0; i < kv.second.sum.size(); ++i) dst[i] += kv.second.sum[i];
    return m->merged_count + m->parked_count;
}

uint32_t ix_merger_finish(ix_merger* m, double* dst, uint64_t len) {
    if (!m || !dst || len != m->pixels * 3) return 0;
    std::lock_guard<std::mutex> lk(m->mu);
    for (auto& kv : m->parked) {
        add_assign(m->merged, kv.second.sum);
        m->merged_count += kv.second.done;
    }
    if (m->budget && !m->parked.empty()) m->budget->release(m->parked.size() * m->pixels * 3 * sizeof(double));
    m->parked.clear();
    m->parked_count = 0;
    if (m->merged.empty()) m->merged.assign(len, 0.0);
    std::memcpy(dst, m->merged.data(), len * sizeof(double));
    return m->merged_count;
}

}  // extern "C"
