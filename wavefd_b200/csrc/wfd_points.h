// Grouping of source/receiver points by the location they write, shared by the single-shot tables
// and the batched ones.
//
// The reference runs its partitions in parallel (no grid point, resp. trace, is shared between
// two partitions: src/spacetime.jl:1087-1129) and each partition sequentially, so every grid cell
// (resp. trace sample) receives its contributions in partition order. A stable sort by the written
// location keeps that order; one thread per group then accumulates it in order.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <vector>

namespace wfd {

template <class T>
struct PointsT {
    long iu, ir;
    T c;
};

// one group per written location: key = 0-based index written, other = 0-based index read
template <class T>
struct Table {
    long npoints = 0, ngroups = 0;
    int by_receiver = 0;
    std::vector<long> key, start, other;
    std::vector<T> c;
    // device copies
    long *d_key = nullptr, *d_start = nullptr, *d_other = nullptr;
    T *d_c = nullptr;
};

template <class T>
void build(Table<T> &t, const std::vector<PointsT<T>> &pts, int by_receiver) {
    t.npoints = (long)pts.size();
    t.by_receiver = by_receiver;
    std::vector<long> order(pts.size());
    std::iota(order.begin(), order.end(), 0L);
    auto keyof = [&](long i) { return by_receiver ? pts[i].ir : pts[i].iu; };
    std::stable_sort(order.begin(), order.end(), [&](long a, long b) { return keyof(a) < keyof(b); });
    t.key.clear();
    t.start.clear();
    t.other.resize(pts.size());
    t.c.resize(pts.size());
    for (size_t j = 0; j < order.size(); j++) {
        const auto &p = pts[order[j]];
        const long k = by_receiver ? p.ir : p.iu;
        if (j == 0 || k != keyof(order[j - 1])) {
            t.key.push_back(k - 1);
            t.start.push_back((long)j);
        }
        t.other[j] = (by_receiver ? p.iu : p.ir) - 1;
        t.c[j] = p.c;
    }
    t.start.push_back((long)order.size());
    t.ngroups = (long)t.key.size();
}

// streaming receiver extraction + forward time interpolation (wfd_interp.cu): one thread per
// receiver group at fine sample jk
void launch_extract_interp(long ngroups, const long *key, const long *start, const long *other, const float *c,
                           const float *field, const float *h, long nh, long jk, long nm, long nd, float *coarse,
                           cudaStream_t s);

}  // namespace wfd
