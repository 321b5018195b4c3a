// scs_window_sort.cuh -- the sigma-window row order of the reference's
// SELL-C-sigma conversion, reproduced exactly on the GPU.
//
// src/utils/convert_formats.hpp:46-55 sorts each sigma window of
// (index, count) pairs with std::sort and the comparator a.count > b.count.
// std::sort is not stable, so rows of equal length are left in whatever
// order the library's algorithm produces.  The reference is built with
// GCC 13.3, whose libstdc++ std::sort is the published introsort restated
// here (the same steps as the C oracle, oracle/smax_oracle.c):
//   sort(a, n):  if n > 0: introsort_loop(0, n, 2*floor(log2 n));
//                          final_insertion_sort(0, n)
//   introsort_loop(lo, hi, depth): while hi - lo > 16:
//       depth == 0 -> heapsort [lo, hi), done;  --depth;
//       move the median of a[lo+1], a[mid], a[hi-1] to a[lo]; Hoare-partition
//       [lo+1, hi) around it at cut; introsort_loop(cut, hi, depth); hi = cut
//   final_insertion_sort: insertion sort of the first 16 entries, then
//       unguarded insertion of the rest (plain insertion sort when n <= 16).
// The order in which disjoint subranges are finished does not change the
// result, so the recursion on [cut, hi) runs from an explicit stack.
//
// Keys: (0x7fffffff - count) << 32 | row, so "a before b" (a.count > b.count)
// is hi32(a) < hi32(b); moving a key moves the row with it.
#pragma once

#include <stdint.h>

namespace smax {
namespace scs_sort {

using Key = unsigned long long;

__device__ __forceinline__ bool before(Key a, Key b) { return (a >> 32) < (b >> 32); }

__device__ __forceinline__ void swap_at(Key *a, int64_t i, int64_t j) {
    const Key t = a[i];
    a[i] = a[j];
    a[j] = t;
}

__device__ inline void median_to_first(Key *a, int64_t r, int64_t x, int64_t y, int64_t z) {
    if (before(a[x], a[y])) {
        if (before(a[y], a[z])) swap_at(a, r, y);
        else if (before(a[x], a[z])) swap_at(a, r, z);
        else swap_at(a, r, x);
    } else if (before(a[x], a[z])) {
        swap_at(a, r, x);
    } else if (before(a[y], a[z])) {
        swap_at(a, r, z);
    } else {
        swap_at(a, r, y);
    }
}

// Hoare partition of [lo, hi) around a[pivot] (pivot = lo - 1).  The median
// of three leaves an entry on each side that stops the scans; the bounds
// tests only keep every access inside the range and never change the result.
__device__ inline int64_t partition(Key *a, int64_t lo, int64_t hi, int64_t pivot) {
    const Key p = a[pivot];
    const int64_t first = lo, last = hi;
    for (;;) {
        while (lo < last - 1 && before(a[lo], p)) ++lo;
        --hi;
        while (hi > first && before(p, a[hi])) --hi;
        if (!(lo < hi)) return lo;
        swap_at(a, lo, hi);
        ++lo;
    }
}

// sift v down from `hole` in the heap a[base .. base+len), then up to `top`
__device__ inline void adjust_heap(Key *a, int64_t base, int64_t hole, int64_t len, Key v) {
    const int64_t top = hole;
    int64_t child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (before(a[base + child], a[base + child - 1])) --child;
        a[base + hole] = a[base + child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[base + hole] = a[base + child - 1];
        hole = child - 1;
    }
    int64_t parent = (hole - 1) / 2;
    while (hole > top && before(a[base + parent], v)) {
        a[base + hole] = a[base + parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[base + hole] = v;
}

__device__ inline void heapsort(Key *a, int64_t lo, int64_t hi) {
    const int64_t len = hi - lo;
    if (len >= 2)
        for (int64_t parent = (len - 2) / 2;; --parent) {
            adjust_heap(a, lo, parent, len, a[lo + parent]);
            if (parent == 0) break;
        }
    for (int64_t last = hi; last - lo > 1;) {
        --last;
        const Key v = a[last];
        a[last] = a[lo];
        adjust_heap(a, lo, 0, last - lo, v);
    }
}

// insertion of a[i] into the sorted a[0..i); a[0] is never after a[i] where
// this is called, so the j >= 0 test only bounds the access
__device__ __forceinline__ void linear_insert(Key *a, int64_t i) {
    const Key v = a[i];
    int64_t j = i - 1;
    while (j >= 0 && before(v, a[j])) {
        a[i] = a[j];
        i = j;
        --j;
    }
    a[i] = v;
}

__device__ inline void insertion_sort(Key *a, int64_t lo, int64_t hi) {
    if (lo == hi) return;
    for (int64_t i = lo + 1; i < hi; ++i) {
        if (before(a[i], a[lo])) {
            const Key v = a[i];
            for (int64_t j = i; j > lo; --j) a[j] = a[j - 1];
            a[lo] = v;
        } else {
            linear_insert(a, i);
        }
    }
}

// Sorts a[0..n) exactly as the reference's std::sort orders its window.
// Returns false if the explicit stack would overflow (never for n < 2^31:
// each pending range has a smaller depth budget than the one before it, so
// at most 2*log2(n) + 1 are pending).
__device__ inline bool std_sort_order(Key *a, int64_t n) {
    if (n <= 0) return true;
    int lg = 0;
    while (((int64_t)1 << (lg + 1)) <= n) ++lg;
    constexpr int kStack = 66;
    int64_t s_lo[kStack], s_hi[kStack];
    int s_depth[kStack];
    int top = 0;
    s_lo[0] = 0;
    s_hi[0] = n;
    s_depth[0] = 2 * lg;
    ++top;
    while (top > 0) {
        --top;
        int64_t lo = s_lo[top], hi = s_hi[top];
        int depth = s_depth[top];
        while (hi - lo > 16) {
            if (depth == 0) {
                heapsort(a, lo, hi);
                break;
            }
            --depth;
            const int64_t mid = lo + (hi - lo) / 2;
            median_to_first(a, lo, lo + 1, mid, hi - 1);
            const int64_t cut = partition(a, lo + 1, hi, lo);
            if (top == kStack) return false;
            s_lo[top] = cut;
            s_hi[top] = hi;
            s_depth[top] = depth;
            ++top;
            hi = cut;
        }
    }
    if (n > 16) {
        insertion_sort(a, 0, 16);
        for (int64_t i = 16; i < n; ++i) linear_insert(a, i);
    } else {
        insertion_sort(a, 0, n);
    }
    return true;
}

}  // namespace scs_sort
}  // namespace smax
