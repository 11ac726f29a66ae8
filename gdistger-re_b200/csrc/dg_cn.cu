// Common-neighbour counts per edge on the device: the job of the reference's
// gcn tool (src/tools/gcn.cpp:249-373), whose output becomes the edge data the
// HuGE transition reads (cn = (int)data, walk.hpp:920).
//
// The tool builds the CSR (both directions with --make-undirected), sorts every
// row by neighbour (duplicates kept), and for each input edge (s, d), in input
// order, computes I = the elements of the shorter of N(s), N(d) (N(s) when they
// are equally long) that occur in the other list, with the shorter list's
// multiplicity, ascending (its galloping search, gcn.cpp:152-197).  Then
// cn = |I|, minus one if I[0] is s or d, and, if cn is still above 1, minus one
// for every later element that repeats its predecessor or is s or d
// (gcn.cpp:327-343).  The value is stored on the first CSR entry (s -> d) and its
// mirror, so every later edge over the same unordered pair reports the value
// computed in the orientation of the pair's first occurrence.
//
// Here: one 64-bit sort builds the row-sorted CSR, a stable sort of the pairs'
// unordered keys finds each pair's first occurrence, one warp per first
// occurrence walks the shorter row and binary-searches the longer one, and the
// counts are scattered back to input order.
#include "dg_internal.h"

#include <cub/cub.cuh>

#include <memory>

namespace {

__global__ void cn_keys(const uint32_t *src, const uint32_t *dst, uint64_t n, int undirected, uint64_t *dir,
                        uint64_t *pair, uint64_t *idx) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t s = src[i], d = dst[i];
        if (undirected) {
            dir[2 * i] = (s << 32) | d;
            dir[2 * i + 1] = (d << 32) | s;
        } else {
            dir[i] = (s << 32) | d;
        }
        pair[i] = s < d ? (s << 32) | d : (d << 32) | s;
        idx[i] = i;
    }
}

__global__ void cn_rows(const uint64_t *dir, uint64_t m, uint32_t v_num, uint64_t *offsets, uint32_t *nbr) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t src = (uint32_t)(dir[i] >> 32);
        const int64_t prev = i == 0 ? -1 : (int64_t)(dir[i - 1] >> 32);
        for (int64_t v = prev + 1; v <= (int64_t)src; v++) offsets[v] = i;
        if (i == m - 1)
            for (uint64_t v = (uint64_t)src + 1; v <= v_num; v++) offsets[v] = m;
        nbr[i] = (uint32_t)dir[i];
    }
}

__device__ __forceinline__ bool in_row(const uint32_t *row, uint64_t len, uint32_t x) {
    uint64_t lo = 0, hi = len;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (row[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo < len && row[lo] == x;
}

// One warp per sorted pair position that starts a group (the pair's first
// occurrence): the count in that occurrence's orientation.
__global__ void cn_count(const uint64_t *pair_sorted, const uint64_t *idx_sorted, uint64_t n, const uint32_t *src,
                         const uint32_t *dst, const uint64_t *offsets, const uint32_t *nbr, int32_t *cn_sorted) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        if (i > 0 && pair_sorted[i] == pair_sorted[i - 1]) continue;
        const uint64_t e = idx_sorted[i];
        const uint32_t s = src[e], d = dst[e];
        const uint32_t *r1 = nbr + offsets[s], *r2 = nbr + offsets[d];
        const uint64_t n1 = offsets[s + 1] - offsets[s], n2 = offsets[d + 1] - offsets[d];
        const bool first_long = n1 > n2;                 // gcn.cpp:166-172
        const uint32_t *sh = first_long ? r2 : r1, *lg = first_long ? r1 : r2;
        const uint64_t ns = first_long ? n2 : n1, nl = first_long ? n1 : n2;
        unsigned long long count = 0, dups = 0, sd = 0;
        uint64_t first = ~0ull;
        if (ns > 0 && nl > 0) {
            for (uint64_t j = lane; j < ns; j += 32) {
                const uint32_t x = sh[j];
                if (!in_row(lg, nl, x)) continue;
                count++;
                first = min(first, j);
                if (j > 0 && sh[j - 1] == x) dups++;
                else if (x == s || x == d) sd++;
            }
        }
        for (int o = 16; o; o >>= 1) {
            count += __shfl_xor_sync(0xffffffffu, count, o);
            dups += __shfl_xor_sync(0xffffffffu, dups, o);
            sd += __shfl_xor_sync(0xffffffffu, sd, o);
            first = min(first, (uint64_t)__shfl_xor_sync(0xffffffffu, (unsigned long long)first, o));
        }
        if (lane == 0) {
            long long c = (long long)count;
            if (c > 0) {
                const uint32_t i0 = sh[first];
                const bool i0_sd = i0 == s || i0 == d;
                if (i0_sd) c--;
                // The first element is never a repeat; an s/d first element was taken off above.
                if (c > 1) c -= (long long)dups + (long long)sd - (i0_sd ? 1 : 0);
            }
            cn_sorted[i] = (int32_t)(uint32_t)c;
        }
    }
}

// Every sorted position takes its group head's count and writes it to input order.
__global__ void cn_scatter(const uint64_t *pair_sorted, const uint64_t *idx_sorted, uint64_t n,
                           const int32_t *cn_sorted, int32_t *cn) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h = i;
        while (h > 0 && pair_sorted[h - 1] == pair_sorted[i]) h--;
        cn[idx_sorted[i]] = cn_sorted[h];
    }
}

template <typename F>
int cub_call(F f) {
    size_t bytes = 0;
    DG_CUDA(f(nullptr, bytes));
    dg::DevArray<uint8_t> tmp;
    DG_CUDA(tmp.alloc(bytes ? bytes : 1));
    DG_CUDA(f(tmp.p, bytes));
    return DG_OK;
}

}  // namespace

extern "C" int dg_common_neighbours(const uint32_t *src, const uint32_t *dst, uint64_t n_edges, uint32_t v_num,
                                    int undirected, int device, int32_t *cn) {
    DG_CHECK(n_edges == 0 || (src && dst && cn), DG_ERR_ARG, "dg_common_neighbours: NULL argument");
    DG_CHECK(v_num > 0, DG_ERR_ARG, "dg_common_neighbours: v_num must be positive");
    for (uint64_t i = 0; i < n_edges; i++)
        DG_CHECK(src[i] < v_num && dst[i] < v_num, DG_ERR_ARG, "edge %llu (%u, %u) has a vertex id >= v_num = %u",
                 (unsigned long long)i, src[i], dst[i], v_num);
    if (n_edges == 0) return DG_OK;
    int n_dev = 0;
    DG_CUDA(cudaGetDeviceCount(&n_dev));
    DG_CHECK(device >= 0 && device < n_dev, DG_ERR_ARG, "device %d out of range (%d)", device, n_dev);
    dg::DeviceGuard guard(device);
    cudaStream_t s = nullptr;
    DG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    } sg{s};
    const uint64_t n = n_edges, m = undirected ? 2 * n : n;
    const unsigned grid = (unsigned)dg::sm_count(device) * 8;
    dg::DevArray<uint32_t> d_src, d_dst, nbr;
    dg::DevArray<uint64_t> dir, dir2, pair, pair2, idx, idx2, offsets;
    dg::DevArray<int32_t> cn_sorted, d_cn;
    DG_CUDA(d_src.alloc(n));
    DG_CUDA(d_dst.alloc(n));
    DG_CUDA(cudaMemcpyAsync(d_src.p, src, n * 4, cudaMemcpyHostToDevice, s));
    DG_CUDA(cudaMemcpyAsync(d_dst.p, dst, n * 4, cudaMemcpyHostToDevice, s));
    DG_CUDA(dir.alloc(m));
    DG_CUDA(dir2.alloc(m));
    DG_CUDA(pair.alloc(n));
    DG_CUDA(pair2.alloc(n));
    DG_CUDA(idx.alloc(n));
    DG_CUDA(idx2.alloc(n));
    cn_keys<<<grid, 256, 0, s>>>(d_src.p, d_dst.p, n, undirected, dir.p, pair.p, idx.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    // Row-sorted CSR (gcn.cpp:130-137 sorts every row by neighbour).
    int rc = cub_call([&](void *t, size_t &b) {
        return cub::DeviceRadixSort::SortKeys(t, b, dir.p, dir2.p, m, 0, 64, s);
    });
    if (rc) return rc;
    DG_CUDA(offsets.alloc((size_t)v_num + 1));
    DG_CUDA(nbr.alloc(m));
    cn_rows<<<grid, 256, 0, s>>>(dir2.p, m, v_num, offsets.p, nbr.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    dir.release();
    dir2.release();
    // Pairs grouped by unordered key, input order kept inside a group (stable sort).
    rc = cub_call([&](void *t, size_t &b) {
        return cub::DeviceRadixSort::SortPairs(t, b, pair.p, pair2.p, idx.p, idx2.p, n, 0, 64, s);
    });
    if (rc) return rc;
    DG_CUDA(cn_sorted.alloc(n));
    DG_CUDA(d_cn.alloc(n));
    cn_count<<<grid, 256, 0, s>>>(pair2.p, idx2.p, n, d_src.p, d_dst.p, offsets.p, nbr.p, cn_sorted.p);
    dg::note_launch();
    cn_scatter<<<grid, 256, 0, s>>>(pair2.p, idx2.p, n, cn_sorted.p, d_cn.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaMemcpyAsync(cn, d_cn.p, n * 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    return DG_OK;
}
