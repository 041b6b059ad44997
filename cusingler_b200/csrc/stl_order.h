// Restatement of the comparison orders of GNU libstdc++'s std::sort and std::minmax_element on
// float with operator<, as host + device code.
//
// The reference sorts each per-label score list with std::sort (src/cusingler.cu:953, inside
// percentile) and picks labels with std::minmax_element (src/cusingler.cu:1123, 1270).  For lists
// without NaN any correct sort or selection gives the same values, and the kernels use a radix
// select.  A constant row makes its correlations NaN (src/cusingler.cu:940-944), and NaN is not
// ordered by operator<, so for NaN-bearing lists the result depends on the exact sequence of
// comparisons and moves.  These routines follow that sequence: introsort with a 16-element
// threshold, median-of-three pivot moved to the front, unguarded Hoare partition, heapsort at depth
// 2*floor(log2 n), then a final insertion sort; and the pairwise min/max scan that keeps the first
// minimum and the last maximum.  They are checked against libstdc++ itself by the test suite.
//
// Where libstdc++ would read outside the array (only possible with NaN breaking its sentinels),
// these routines stop at the array bound instead and set *oob = 1.
#pragma once

#include <cstdint>

#ifndef SGR_HD
#if defined(__CUDACC__)
#define SGR_HD __host__ __device__
#else
#define SGR_HD
#endif
#endif

namespace sgr {
namespace stl {

SGR_HD inline void swapf(float* a, int i, int j) {
    float t = a[i];
    a[i] = a[j];
    a[j] = t;
}

SGR_HD inline int floor_log2(int n) {
    int r = 0;
    while (n > 1) {
        n >>= 1;
        ++r;
    }
    return r;
}

// Sift `value` down from `hole` in the max-heap a[0..len), then back up towards `top`.
SGR_HD inline void heap_adjust(float* a, int hole, int len, float value) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (a[child] < a[child - 1]) child--;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > top && a[parent] < value) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = value;
}

SGR_HD inline void heap_sort(float* a, int len) {
    if (len >= 2) {
        for (int parent = (len - 2) / 2;; --parent) {
            heap_adjust(a, parent, len, a[parent]);
            if (parent == 0) break;
        }
    }
    for (int last = len; last > 1;) {
        --last;
        float v = a[last];
        a[last] = a[0];
        heap_adjust(a, 0, last, v);
    }
}

// Pivot selection (median of a[f+1], a[mid], a[l-1] moved to a[f]) and partition of (f, l).
SGR_HD inline int partition_pivot(float* a, int f, int l, int* oob) {
    int mid = f + (l - f) / 2;
    int x = f + 1, y = mid, z = l - 1;
    if (a[x] < a[y]) {
        if (a[y] < a[z]) swapf(a, f, y);
        else if (a[x] < a[z]) swapf(a, f, z);
        else swapf(a, f, x);
    } else if (a[x] < a[z]) {
        swapf(a, f, x);
    } else if (a[y] < a[z]) {
        swapf(a, f, z);
    } else {
        swapf(a, f, y);
    }
    const float pivot = a[f];
    int lo = f + 1, hi = l;
    for (;;) {
        while (a[lo] < pivot) {
            ++lo;
            if (lo >= l) {
                *oob = 1;
                return l - 1;
            }
        }
        --hi;
        while (pivot < a[hi]) {
            --hi;
            if (hi <= f) {
                *oob = 1;
                return f + 1;
            }
        }
        if (!(lo < hi)) return lo;
        swapf(a, lo, hi);
        ++lo;
    }
}

// Insertion of a[i] into the sorted prefix without a lower guard (libstdc++'s unguarded insert);
// the bound check only reports what libstdc++ would have read past.
SGR_HD inline void linear_insert(float* a, int i, int* oob) {
    float v = a[i];
    int j = i - 1;
    while (v < a[j]) {
        a[j + 1] = a[j];
        --j;
        if (j < 0) {
            *oob = 1;
            break;
        }
    }
    a[j + 1] = v;
}

SGR_HD inline void guarded_insertion_sort(float* a, int f, int l, int* oob) {
    for (int i = f + 1; i < l; ++i) {
        if (a[i] < a[f]) {
            float v = a[i];
            for (int j = i; j > f; --j) a[j] = a[j - 1];
            a[f] = v;
        } else {
            linear_insert(a, i, oob);
        }
    }
}

// std::sort(a, a + n).  Uses an explicit stack; subranges are disjoint, so the order in which
// they are finished does not change the result.
SGR_HD inline void sort(float* a, int n, int* oob) {
    const int threshold = 16;
    if (n <= 1) return;
    struct Range { int f, l, depth; };
    Range stack[64];
    int sp = 0;
    stack[sp++] = {0, n, 2 * floor_log2(n)};
    while (sp > 0) {
        Range r = stack[--sp];
        int f = r.f, l = r.l, depth = r.depth;
        while (l - f > threshold) {
            if (depth == 0) {
                heap_sort(a + f, l - f);
                break;
            }
            --depth;
            int cut = partition_pivot(a, f, l, oob);
            if (sp < 64) stack[sp++] = {cut, l, depth};
            else *oob = 1;
            l = cut;
        }
    }
    if (n > threshold) {
        guarded_insertion_sort(a, 0, threshold, oob);
        for (int i = threshold; i < n; ++i) linear_insert(a, i, oob);
    } else {
        guarded_insertion_sort(a, 0, n, oob);
    }
}

// std::minmax_element(v, v + n) as index pair (first minimum, last maximum).
SGR_HD inline void minmax(const float* v, int n, int* mn, int* mx) {
    if (n <= 1) {
        *mn = 0;
        *mx = 0;
        return;
    }
    int lo, hi;
    if (v[1] < v[0]) {
        lo = 1;
        hi = 0;
    } else {
        lo = 0;
        hi = 1;
    }
    int i = 2;
    while (i < n) {
        if (i + 1 == n) {
            if (v[i] < v[lo]) lo = i;
            else if (!(v[i] < v[hi])) hi = i;
            break;
        }
        if (v[i + 1] < v[i]) {
            if (v[i + 1] < v[lo]) lo = i + 1;
            if (!(v[i] < v[hi])) hi = i;
        } else {
            if (v[i] < v[lo]) lo = i;
            if (!(v[i + 1] < v[hi])) hi = i + 1;
        }
        i += 2;
    }
    *mn = lo;
    *mx = hi;
}

}  // namespace stl
}  // namespace sgr
