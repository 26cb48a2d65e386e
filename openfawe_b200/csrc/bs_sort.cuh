// Device-wide exclusive scan and stable LSD radix sort (project-written; used by the tree builds).
#pragma once
#include "bs_internal.cuh"

namespace bs {

// out[i] = sum(in[0..i)); *total (device, may be null) = sum(in[0..n)).  in and out may alias.
int scan_exclusive(const int64_t *in, int64_t *out, int64_t n, int64_t *total, Scratch &scratch, cudaStream_t s);

// Stable sort of (keys, vals) by key bits [begin_bit, end_bit) (8-bit digits: the last one may take bits above
// end_bit); results back in keys/vals.
int radix_sort(uint64_t *keys, int32_t *vals, int64_t n, int begin_bit, int end_bit, Scratch &scratch,
               cudaStream_t s);

// After the stream has synchronised: BS_OK, or an error if a sort since the last check gave up waiting on the
// look-back of an earlier tile (its order is then invalid).  Clears the record.
int check_sort_fault();
// The fault flag's device address (null if it cannot be had), for a copy queued with a call's other results; and the
// check of a flag value read that way (clears the flag and reports the fault, as check_sort_fault).
const int *sort_fault_flag();
int sort_fault_seen(int fault);

}  // namespace bs
