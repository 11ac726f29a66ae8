/*
 * Stand-in for the un-vendored hnswlib dependency of src/word2vec.cu
 * (ext/hnswlib is an empty directory in the reference; word2vec.cu:18 includes
 * "hnswlib.h").  word2vec.cu uses it only in its evaluation helper
 * count_ann_intersection (word2vec.cu:1144-1204), never on the training path,
 * so every member is a no-op and searches return nothing.  Project-written test
 * infrastructure: it lets the reference's own CUDA kernels compile unmodified
 * into oracle/_ref/ as the checker of the SGNS restatement.
 */
#ifndef DG_REF_SHIM_HNSWLIB_H
#define DG_REF_SHIM_HNSWLIB_H

#include <cstddef>
#include <queue>
#include <utility>

namespace hnswlib {

typedef size_t labeltype;

class L2Space {
public:
    explicit L2Space(size_t dim) : dim_(dim) {}
    size_t dim_;
};

template <typename dist_t>
class HierarchicalNSW {
public:
    HierarchicalNSW(L2Space *, size_t, size_t = 16, size_t = 200) {}
    void addPoint(const void *, labeltype) {}
    std::priority_queue<std::pair<dist_t, labeltype>> searchKnn(const void *, size_t) const {
        return std::priority_queue<std::pair<dist_t, labeltype>>();
    }
};

}  // namespace hnswlib

#endif
