// Introsort exactly as the GNU C++ library's std::sort performs it, for the
// three places where the reference sorts Neighbor records by distance alone
// and the order of equal-distance records is therefore fixed by the library's
// algorithm, not by the data:
//   kgraph.cpp:476  sort(knn.begin(), knn.begin() + L)   -- search seed pool
//   kgraph.cpp:697  std::sort(v.begin(), v.end())         -- reverse edges
//   kgraph.cpp:793  sort(pool.begin(), pool.begin() + L)  -- build init pool
// Reproducing the same permutation on the GPU keeps search bit-identical to
// the reference even when distances tie (integer-valued data ties often).
//
// The algorithm is the published introsort (Musser 1997) with the GNU
// choices: depth limit 2*floor(log2 n); partitions while more than 16
// elements remain, recursing on the right part; median-of-three of
// (first+1, mid, last-1) moved to first; unguarded Hoare partition; heapsort
// (make_heap + sort_heap) when the depth limit is spent; a final insertion
// sort (guarded for the first 16, unguarded after).  Comparisons are `a < b`
// on the key only.
//
// Written as a template over an accessor so the same code runs in a CUDA
// thread (device) and in the host tests that check it against std::sort.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define KG_HD __host__ __device__ __forceinline__
#else
#define KG_HD inline
#endif

namespace kgb {

// A: struct with  float key(int i); void swap(int i, int j);
//                 Rec get(int i); void put(int i, Rec r); float rkey(Rec r)
template <typename A>
KG_HD void gs_move_median_to_first(A &a, int result, int x, int y, int z) {
    if (a.key(x) < a.key(y)) {
        if (a.key(y) < a.key(z)) a.swap(result, y);
        else if (a.key(x) < a.key(z)) a.swap(result, z);
        else a.swap(result, x);
    } else if (a.key(x) < a.key(z)) a.swap(result, x);
    else if (a.key(y) < a.key(z)) a.swap(result, z);
    else a.swap(result, y);
}

template <typename A>
KG_HD int gs_unguarded_partition(A &a, int first, int last, int pivot) {
    while (true) {
        while (a.key(first) < a.key(pivot)) ++first;
        --last;
        while (a.key(pivot) < a.key(last)) --last;
        if (!(first < last)) return first;
        a.swap(first, last);
        ++first;
    }
}

template <typename A, typename R>
KG_HD void gs_push_heap(A &a, int first, int hole, int top, R value) {
    int parent = (hole - 1) / 2;
    while (hole > top && a.key(first + parent) < a.rkey(value)) {
        a.put(first + hole, a.get(first + parent));
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a.put(first + hole, value);
}

template <typename A, typename R>
KG_HD void gs_adjust_heap(A &a, int first, int hole, int len, R value) {
    const int top = hole;
    int second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (a.key(first + second) < a.key(first + (second - 1))) second--;
        a.put(first + hole, a.get(first + second));
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        a.put(first + hole, a.get(first + (second - 1)));
        hole = second - 1;
    }
    gs_push_heap(a, first, hole, top, value);
}

template <typename A>
KG_HD void gs_heapsort(A &a, int first, int last) {
    int len = last - first;
    if (len >= 2) {   // make_heap
        int parent = (len - 2) / 2;
        while (true) {
            auto v = a.get(first + parent);
            gs_adjust_heap(a, first, parent, len, v);
            if (parent == 0) break;
            parent--;
        }
    }
    while (last - first > 1) {   // sort_heap: pop_heap(first, last, last)
        --last;
        auto v = a.get(last);
        a.put(last, a.get(first));
        gs_adjust_heap(a, first, 0, last - first, v);
    }
}

template <typename A>
KG_HD void gs_unguarded_linear_insert(A &a, int last) {
    auto val = a.get(last);
    int next = last - 1;
    while (a.rkey(val) < a.key(next)) {
        a.put(last, a.get(next));
        last = next;
        --next;
    }
    a.put(last, val);
}

template <typename A>
KG_HD void gs_insertion_sort(A &a, int first, int last) {
    if (first == last) return;
    for (int i = first + 1; i != last; ++i) {
        if (a.key(i) < a.key(first)) {
            auto val = a.get(i);
            for (int j = i; j > first; --j) a.put(j, a.get(j - 1));
            a.put(first, val);
        } else {
            gs_unguarded_linear_insert(a, i);
        }
    }
}

KG_HD int gs_lg(int n) {
    int r = 0;
    while (n > 1) { n >>= 1; ++r; }
    return r;
}

template <typename A>
KG_HD void gnu_sort(A &a, int first, int last) {
    if (first == last) return;
    // __introsort_loop with an explicit stack.  The recursive form is
    //   while (n > 16) { if (!depth) heapsort, return; --depth;
    //                    cut = partition; recurse(cut, last, depth); last = cut; }
    // so the right part is finished before the left part continues with the
    // same (decremented) depth: the left frame is pushed under the right one.
    struct Frame { int first, last, depth; };
    Frame stack[72];
    int sp = 0;
    stack[sp++] = Frame{first, last, gs_lg(last - first) * 2};
    while (sp > 0) {
        Frame f = stack[--sp];
        if (f.last - f.first <= 16) continue;
        if (f.depth == 0) { gs_heapsort(a, f.first, f.last); continue; }
        int depth = f.depth - 1;
        int mid = f.first + (f.last - f.first) / 2;
        gs_move_median_to_first(a, f.first, f.first + 1, mid, f.last - 1);
        int cut = gs_unguarded_partition(a, f.first + 1, f.last, f.first);
        stack[sp++] = Frame{f.first, cut, depth};
        stack[sp++] = Frame{cut, f.last, depth};
    }
    // __final_insertion_sort
    if (last - first > 16) {
        gs_insertion_sort(a, first, first + 16);
        for (int i = first + 16; i != last; ++i) gs_unguarded_linear_insert(a, i);
    } else {
        gs_insertion_sort(a, first, last);
    }
}

}  // namespace kgb
