/*
 * ix_dispatch.h -- host-side sample-range dispatch and deterministic merge.
 *
 * The reference's indicatrix-dispatch (crates/indicatrix-dispatch) splits one image's
 * absolute sample range across lanes (CPU threads, GPUs, remote workers) and merges the
 * lanes' per-pixel sums so the result does not depend on which lane traced which chunk
 * or in which order the chunks finished.  These are the two pieces of it a multi-GPU
 * or multi-process run of this backend needs, in C for any host language:
 *
 *   ix_sample_cursor  -- SampleCursor (sample_cursor/mod.rs:64-230): disjoint absolute
 *                        sample ranges handed out in order; failed chunks re-queued.
 *   ix_merger         -- Merger (merge/mod.rs:155-330): a left fold of chunk sums in
 *                        ascending first-sample order; chunks arriving ahead of the
 *                        frontier are parked; invalid pixels (non-finite or negative)
 *                        are zeroed and counted; a parked-memory budget bounds parking.
 * Sums are f64 here (the reference folds f32 Vec3).  Thread-safe.
 */
#ifndef IX_DISPATCH_H
#define IX_DISPATCH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ix_sample_cursor ix_sample_cursor;
/* SampleCursor::new(start, end). */
ix_sample_cursor* ix_sample_cursor_new(uint32_t start, uint32_t end);
void ix_sample_cursor_free(ix_sample_cursor* c);
/* SampleCursor::claim (sample_cursor/mod.rs:119): re-queued ranges first, then the next
 * `want` samples; returns 1 and the range, or 0 when everything is claimed. */
int ix_sample_cursor_claim(ix_sample_cursor* c, uint32_t want, uint32_t* start, uint32_t* count);
/* SampleCursor::requeue (:218): a failed lane's chunk goes back to be claimed again. */
void ix_sample_cursor_requeue(ix_sample_cursor* c, uint32_t start, uint32_t count);
/* SampleCursor::fully_claimed (:188). */
int ix_sample_cursor_fully_claimed(const ix_sample_cursor* c);

enum { IX_MERGE_OK = 0, IX_MERGE_WRONG_LENGTH = -1, IX_MERGE_OVERLAP = -2,
       IX_MERGE_BUDGET = -3 };
typedef struct ix_merger ix_merger;
/* Merger::new(pixels, first_sample) with a parked-memory budget of its own in bytes
 * (0 = none). */
ix_merger* ix_merger_new(uint64_t pixels, uint32_t first_sample, uint64_t parked_budget_bytes);
/* A byte budget shared by several mergers (ParkedBudget, merge/mod.rs:72-80): each parked
 * chunk reserves pixels * 24 bytes from it and releases them when the chunk folds, when
 * ix_merger_finish runs, or when its merger is freed with the chunk still parked.
 * Thread-safe; free it after every merger that uses it. */
typedef struct ix_parked_budget ix_parked_budget;
ix_parked_budget* ix_parked_budget_new(uint64_t bytes);
void ix_parked_budget_free(ix_parked_budget* b);
uint64_t ix_parked_budget_used(ix_parked_budget* b);
/* Merger::new(pixels, first_sample).with_parked_budget(budget) (merge/mod.rs:190). */
ix_merger* ix_merger_new_shared(uint64_t pixels, uint32_t first_sample, ix_parked_budget* budget);
void ix_merger_free(ix_merger* m);
/* Merger::add (merge/mod.rs:239): chunk [first_sample, first_sample + done) with its
 * per-pixel sums (`len` doubles = pixels * 3).  *total (may be NULL) receives the
 * samples merged or parked so far. */
int ix_merger_add(ix_merger* m, uint32_t first_sample, uint32_t done, const double* sums,
                  uint64_t len, uint32_t* total);
uint32_t ix_merger_frontier(const ix_merger* m);
uint32_t ix_merger_total(const ix_merger* m);
uint64_t ix_merger_dropped_pixels(const ix_merger* m);
/* Merger::snapshot_into (:300): adds merged + parked sums into dst; returns the count. */
uint32_t ix_merger_snapshot(const ix_merger* m, double* dst, uint64_t len);
/* Merger::into_parts (:319): folds parked chunks in order, writes the merged sums to
 * dst (overwriting) and returns the merged sample count. */
uint32_t ix_merger_finish(ix_merger* m, double* dst, uint64_t len);

#ifdef __cplusplus
}
#endif
#endif
