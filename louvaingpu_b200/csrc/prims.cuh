// Device-wide primitives written for this library (no CUB/Thrust): exclusive
// scans, the fixed-tree FP64 sum and a stable LSD radix sort of
// (64-bit key, float payload) pairs.
#pragma once
#include "lvg_internal.cuh"

namespace lvg {

// out[0..n] = exclusive scan of in[0..n), out[n] = total.  out may alias in
// (then in needs n+1 entries).  Scratch comes from the arena's high end.
void scan_u32(const uint32_t* in, uint32_t* out, int64_t n, Arena& a, cudaStream_t s);
void scan_i64(const int64_t* in, int64_t* out, int64_t n, Arena& a, cudaStream_t s);

// Fixed-tree sum (see lvg_internal.cuh) of n doubles or floats into *d_out.
void tree_sum_f64(const double* x, int64_t n, double* d_out, Arena& a, cudaStream_t s);
void tree_sum_f32(const float* x, int64_t n, double* d_out, Arena& a, cudaStream_t s);
// Reduce `n` group partials (already produced by a group_sum_block pass) to
// one value in *d_out.
void tree_finish(const double* partials, int64_t n, double* d_out, Arena& a, cudaStream_t s);

// Stable sort of (keys, vals) by the low `bits` bits of the keys.  The data
// moves between (k0, v0) and (k1, v1); the return value says which pair holds
// the result (0 or 1).  Requires n < 2^32.
int radix_sort_pairs(uint64_t* k0, float* v0, uint64_t* k1, float* v1, int64_t n, int bits, Arena& a,
                     cudaStream_t s);
// The same, by key bits [lo, lo + bits): the bits below lo ride along, the
// bits from lo + bits up must be zero (the last 8-bit digit reads them).
int radix_sort_pairs_range(uint64_t* k0, float* v0, uint64_t* k1, float* v1, int64_t n, int lo, int bits, Arena& a,
                           cudaStream_t s);

}  // namespace lvg
