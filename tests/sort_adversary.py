"""Inputs that drive the reference's window sort into its heapsort fallback.

The SELL-C-sigma conversion orders each sigma window with std::sort; the
oracle (oracle/smax_oracle.c) and the GPU (csrc/scs_window_sort.cuh) restate
GCC 13.3 libstdc++'s introsort so the order of equal-length rows is the
reference's.  Random row lengths never exhaust introsort's depth budget
(2*floor(log2 n) partitions), so the heapsort branch needs a crafted input.

`sort_steps` is a Python statement of the same introsort control flow (no
final insertion pass: only the partition sequence matters here) with a
pluggable comparison; `adversary(n)` runs it against McIlroy's adversary
("A Killer Adversary for Quicksort", Software: Practice and Experience
29(4), 1999), which fixes element values lazily so that every partition is
as unbalanced as possible.  The values it returns are a fixed input on which
the same steps reach the heapsort fallback; `uses_heap` checks that for any
input.  Test infrastructure only.
"""
from __future__ import annotations


def sort_steps(n: int, before) -> bool:
    """Runs introsort's partition steps on items 0..n-1 with the strict order
    `before(i, j)`; returns True if some range fell back to heapsort."""
    a = list(range(n))
    heap = False

    def sw(i, j):
        a[i], a[j] = a[j], a[i]

    def median_to_first(r, x, y, z):
        if before(a[x], a[y]):
            if before(a[y], a[z]):
                sw(r, y)
            elif before(a[x], a[z]):
                sw(r, z)
            else:
                sw(r, x)
        elif before(a[x], a[z]):
            sw(r, x)
        elif before(a[y], a[z]):
            sw(r, z)
        else:
            sw(r, y)

    def partition(lo, hi, p):
        while True:
            while before(a[lo], a[p]):
                lo += 1
            hi -= 1
            while before(a[p], a[hi]):
                hi -= 1
            if not lo < hi:
                return lo
            sw(lo, hi)
            lo += 1

    stack = [(0, n, 2 * (n.bit_length() - 1))] if n > 0 else []
    while stack:
        lo, hi, depth = stack.pop()
        while hi - lo > 16:
            if depth == 0:
                heap = True
                break
            depth -= 1
            median_to_first(lo, lo + 1, lo + (hi - lo) // 2, hi - 1)
            cut = partition(lo + 1, hi, lo)
            stack.append((cut, hi, depth))
            hi = cut
    return heap


def adversary(n: int) -> list[int]:
    """McIlroy's adversary: values (smaller = earlier in the sorted order) on
    which introsort's partitions degenerate."""
    gas = n
    val = [gas] * n
    state = {"solid": 0, "cand": 0}

    def freeze(i):
        val[i] = state["solid"]
        state["solid"] += 1

    def before(i, j):
        if val[i] == gas and val[j] == gas:
            freeze(i if i == state["cand"] else j)
        if val[i] == gas:
            state["cand"] = i
        elif val[j] == gas:
            state["cand"] = j
        return val[i] < val[j]

    sort_steps(n, before)
    for i in range(n):
        if val[i] == gas:
            freeze(i)
    return val


def uses_heap(values) -> bool:
    return sort_steps(len(values), lambda i, j: values[i] < values[j])


def heap_row_lengths(n: int) -> list[int]:
    """Row lengths for one sigma window of n rows that reach the heapsort
    fallback with many equal lengths (adversary values paired up: v // 2).
    Longer rows sort first, so length = max - v//2 + 1."""
    v = [x // 2 for x in adversary(n)]
    top = max(v)
    return [top - x + 1 for x in v]
