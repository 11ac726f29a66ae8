// Graph loading: binary edge records -> device CSR with per-entry acceptance
// thresholds, plus the entropy-term table the walk kernel reads.
#include "dg_internal.h"

#include <cub/cub.cuh>

#include <cerrno>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>

namespace {

constexpr uint32_t kRandMax = 2147483647u;  // glibc RAND_MAX, walk.hpp:928
constexpr uint32_t kNever = 0x80000000u;    // threshold no 31-bit draw reaches

struct HostEdge {
    uint32_t src, dst;
    float data;
};
static_assert(sizeof(HostEdge) == 12, "edge records are 12 bytes (storage.hpp:15-37)");

// Smallest k in [0, 2^31 - 1] with t <= k / 2147483647.0, the draw at which the
// reference's `p_norm <= p` (walk.hpp:938) first holds.  The guess is within one
// or two of the answer; the corrections are capped for safety.
__device__ uint32_t threshold_of(double t) {
    if (isnan(t)) return kNever;
    if (t <= 0.0) return 0u;
    if (t > 1.0) return kNever;
    long long k = (long long)ceil(__dmul_rn(t, (double)kRandMax));
    if (k > (long long)kRandMax) k = kRandMax;
    if (k < 0) k = 0;
    for (int i = 0; i < 64 && k > 0 && t <= __ddiv_rn((double)(k - 1), (double)kRandMax); i++) k--;
    for (int i = 0; i < 64 && k <= (long long)kRandMax && !(t <= __ddiv_rn((double)k, (double)kRandMax)); i++) k++;
    return k > (long long)kRandMax ? kNever : (uint32_t)k;
}

// One warp per source vertex: p_accept = (1 / (sd - cn)) * max(sd, dd) / min(sd, dd),
// p_norm = tanh(p_accept) (walk.hpp:920-934), folded into an integer threshold so
// that the walk's accept test is a single compare against its 31-bit draw.
__global__ void threshold_kernel(const uint64_t *__restrict__ offsets, const uint32_t *__restrict__ nbr,
                                 const float *__restrict__ data, const uint32_t *__restrict__ deg,
                                 uint32_t v_num, uint2 *__restrict__ entries) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = warp; v < v_num; v += n_warps) {
        const int sd = (int)deg[v];
        const uint64_t end = offsets[v + 1];
        for (uint64_t e = offsets[v] + lane; e < end; e += 32) {
            const uint32_t dst = nbr[e];
            const int cn = __float2int_rz(data[e]);
            const int dd = (int)deg[dst];
            const int hi = sd > dd ? sd : dd, lo = sd < dd ? sd : dd;
            const double p_accept =
                __ddiv_rn(__dmul_rn(__ddiv_rn(1.0, (double)(sd - cn)), (double)hi), (double)lo);
            entries[e] = make_uint2(dst, threshold_of(tanh(p_accept)));
        }
    }
}

// Correlation::SnSn_div_Snp1Snp1 / FjFj_div_FiFi / iterateHn (walk.hpp:284-304):
// the log2 term depends only on the integers (Sn, fi), so the host tabulates it
// once with the C library's pow/log2 -- the same functions the reference calls.
double entropy_term(double Sn, double fi) {
    const double k = 1.0;
    double Snp1 = Sn + k;
    double a = std::pow(Sn / Snp1, Sn) * std::pow(1.0 / Snp1, k);
    if (fi == 0) return std::log2(a);
    double fj = fi + k;
    double b = std::pow(fj / fi, fi) * std::pow(fj, k);
    return std::log2(a * b);
}

// First record (lowest index) that the reference would reject: a vertex id >=
// v_num (graph.hpp:639 asserts) or data the transition's (int) conversion cannot
// hold (walk.hpp:920).
__global__ void check_records(const HostEdge *__restrict__ e, uint64_t n, uint32_t v_num, unsigned long long *bad) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const HostEdge r = e[i];
        const bool ok = r.src < v_num && r.dst < v_num && isfinite(r.data) && r.data > -2147483648.0f &&
                        r.data < 2147483648.0f;
        if (!ok) atomicMin(bad, (unsigned long long)i);
    }
}

// CSR entries in emission order: record i gives entry i (directed) or entries 2i
// (src -> dst) and 2i + 1 (dst -> src) (graph.hpp:671-686); row = source, value
// = data bits << 32 | neighbour.  Degrees are counted on the way.
__global__ void emit_entries(const HostEdge *__restrict__ e, uint64_t n, int undirected, uint32_t *rows,
                             unsigned long long *vals, uint32_t *out_deg, uint32_t *in_deg) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const HostEdge r = e[i];
        const unsigned long long bits = (unsigned long long)__float_as_uint(r.data) << 32;
        const uint64_t k = undirected ? 2 * i : i;
        rows[k] = r.src;
        vals[k] = bits | r.dst;
        atomicAdd(&out_deg[r.src], 1u);
        atomicAdd(&in_deg[r.dst], 1u);
        if (undirected) {
            rows[k + 1] = r.dst;
            vals[k + 1] = bits | r.src;
            atomicAdd(&out_deg[r.dst], 1u);
            atomicAdd(&in_deg[r.src], 1u);
        }
    }
}

__global__ void split_values(const unsigned long long *__restrict__ vals, uint64_t m, uint32_t *nbr, float *data) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long v = vals[k];
        nbr[k] = (uint32_t)v;
        data[k] = __uint_as_float((uint32_t)(v >> 32));
    }
}

// Loaded records to the device CSR, all on the device: validation, doubling,
// a stable radix sort of the entries by source row (so each row keeps record
// order, the reference's bucketing, graph.hpp:509-540), degrees, offsets,
// then the acceptance thresholds.
int build_graph(const HostEdge *edges, uint64_t n_edges, uint32_t v_num, int undirected, int device,
                dg_graph **out) {
    DG_CHECK(out != nullptr, DG_ERR_ARG, "dg_graph_create: out is NULL");
    *out = nullptr;
    DG_CHECK(v_num > 0, DG_ERR_ARG, "dg_graph_create: v_num must be positive");
    int n_dev = 0;
    DG_CUDA(cudaGetDeviceCount(&n_dev));
    DG_CHECK(device >= 0 && device < n_dev, DG_ERR_ARG, "dg_graph_create: device %d out of range (%d)", device, n_dev);
    const uint64_t m = undirected ? 2 * n_edges : n_edges;
    DG_CHECK(m < (1ull << 40), DG_ERR_ARG, "too many edges");

    dg::DeviceGuard guard(device);
    std::unique_ptr<dg_graph> g(new dg_graph());
    g->device = device;
    g->v_num = v_num;
    g->m = m;
    DG_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    cudaStream_t s = g->stream;
    const unsigned grid = (unsigned)dg::sm_count(device) * 8;
    DG_CUDA(g->offsets.alloc((size_t)v_num + 1));
    DG_CUDA(g->entries.alloc(m));
    DG_CUDA(g->out_deg.alloc(v_num));
    DG_CUDA(g->in_deg.alloc(v_num));
    DG_CUDA(g->freq.alloc(v_num));
    DG_CUDA(cudaMemsetAsync(g->freq.p, 0, (size_t)v_num * 4, s));
    DG_CUDA(cudaMemsetAsync(g->out_deg.p, 0, (size_t)v_num * 4, s));
    DG_CUDA(cudaMemsetAsync(g->in_deg.p, 0, (size_t)v_num * 4, s));
    if (n_edges) {
        dg::DevArray<HostEdge> rec;
        DG_CUDA(rec.alloc(n_edges));
        DG_CUDA(cudaMemcpyAsync(rec.p, edges, n_edges * sizeof(HostEdge), cudaMemcpyHostToDevice, s));
        dg::DevArray<unsigned long long> bad;
        DG_CUDA(bad.alloc(1));
        DG_CUDA(cudaMemsetAsync(bad.p, 0xFF, sizeof(unsigned long long), s));
        check_records<<<grid, 256, 0, s>>>(rec.p, n_edges, v_num, bad.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
        unsigned long long first_bad = 0;
        DG_CUDA(cudaMemcpyAsync(&first_bad, bad.p, sizeof(first_bad), cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        if (first_bad != ~0ull) {
            const HostEdge &e = edges[first_bad];
            if (!(e.src < v_num && e.dst < v_num))
                return dg::fail(DG_ERR_ARG, "edge %llu (%u, %u) has a vertex id >= v_num = %u", first_bad, e.src,
                                e.dst, v_num);
            return dg::fail(DG_ERR_ARG, "edge %llu has data %g outside the int range the transition converts it to",
                            first_bad, (double)e.data);
        }
        dg::DevArray<uint32_t> rows, rows_alt;
        dg::DevArray<unsigned long long> vals, vals_alt;
        DG_CUDA(rows.alloc(m));
        DG_CUDA(vals.alloc(m));
        emit_entries<<<grid, 256, 0, s>>>(rec.p, n_edges, undirected, rows.p, vals.p, g->out_deg.p, g->in_deg.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaStreamSynchronize(s));
        rec.release();
        DG_CUDA(rows_alt.alloc(m));
        DG_CUDA(vals_alt.alloc(m));
        cub::DoubleBuffer<uint32_t> kb(rows.p, rows_alt.p);
        cub::DoubleBuffer<unsigned long long> vb(vals.p, vals_alt.p);
        const int end_bit = v_num > 1 ? 32 - __builtin_clz(v_num - 1) : 1;
        {
            size_t bytes = 0;
            DG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, m, 0, end_bit, s));
            dg::DevArray<uint8_t> tmp;
            DG_CUDA(tmp.alloc(bytes ? bytes : 1));
            DG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, kb, vb, m, 0, end_bit, s));
            DG_CUDA(cudaStreamSynchronize(s));
        }
        if (vb.Current() != vals.p) vals.swap(vals_alt);
        rows.release();
        rows_alt.release();
        // vals_alt (m x 8 bytes) holds the neighbour and data columns.
        uint32_t *nbr = reinterpret_cast<uint32_t *>(vals_alt.p);
        float *data = reinterpret_cast<float *>(vals_alt.p) + m;
        split_values<<<grid, 256, 0, s>>>(vals.p, m, nbr, data);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
        int rc = dg::exclusive_scan_u32_to_u64(g->out_deg.p, g->offsets.p, v_num, s);
        if (rc) return rc;
        vals.release();
        dg::EventTimer t;
        t.start(s);
        threshold_kernel<<<grid, 256, 0, s>>>(g->offsets.p, nbr, data, g->out_deg.p, v_num, g->entries.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
        t.stop(s);
        DG_CUDA(cudaStreamSynchronize(s));
        g->threshold_ms = t.ms();
    } else {
        DG_CUDA(cudaMemsetAsync(g->offsets.p, 0, ((size_t)v_num + 1) * 8, s));
    }
    g->h_out_deg.resize(v_num);
    DG_CUDA(cudaMemcpyAsync(g->h_out_deg.data(), g->out_deg.p, (size_t)v_num * 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    *out = g.release();
    return DG_OK;
}

}  // namespace

dg_graph::~dg_graph() {
    if (stream) {
        dg::DeviceGuard guard(device);
        cudaStreamSynchronize(stream);
        offsets.release();
        entries.release();
        out_deg.release();
        in_deg.release();
        freq.release();
        etable.release();
        cudaStreamDestroy(stream);
    }
}

namespace dg {

int ensure_entropy_table(dg_graph *g, uint32_t max_sn) {
    if (g->etable_max_sn >= max_sn && g->etable.p) return DG_OK;
    const uint64_t n = (uint64_t)max_sn * (max_sn + 1) / 2 + max_sn;
    std::vector<double> t(n);
    for (uint32_t s = 1; s <= max_sn; s++)
        for (uint32_t f = 0; f <= s; f++) t[(uint64_t)s * (s + 1) / 2 + f - 1] = entropy_term((double)s, (double)f);
    DG_CUDA(g->etable.alloc(n));
    DG_CUDA(cudaMemcpyAsync(g->etable.p, t.data(), n * 8, cudaMemcpyHostToDevice, g->stream));
    DG_CUDA(cudaStreamSynchronize(g->stream));
    g->etable_max_sn = max_sn;
    return DG_OK;
}

}  // namespace dg

extern "C" int dg_graph_create_from_edges(const void *edges, uint64_t n_edges, uint32_t v_num, int undirected,
                                          int device, dg_graph **out) {
    DG_CHECK(edges != nullptr || n_edges == 0, DG_ERR_ARG, "dg_graph_create_from_edges: edges is NULL");
    return build_graph(static_cast<const HostEdge *>(edges), n_edges, v_num, undirected, device, out);
}

// ------------------------------------------------- CSR from device edges

namespace {

__global__ void double_keys(const uint64_t *keys, uint64_t n, uint64_t *out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        out[2 * i] = k;
        out[2 * i + 1] = (k << 32) | (k >> 32);
    }
}

// Row offsets of sorted directed keys (src in the high word), then the
// neighbour and edge-data columns.
__global__ void csr_columns(const uint64_t *d, uint64_t m, uint32_t v_num, uint64_t data_seed, int weighted,
                            uint64_t *offsets, uint32_t *nbr, float *data) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t src = (uint32_t)(d[i] >> 32), dst = (uint32_t)d[i];
        const int64_t prev = i == 0 ? -1 : (int64_t)(d[i - 1] >> 32);
        for (int64_t v = prev + 1; v <= (int64_t)src; v++) offsets[v] = i;
        if (i == m - 1)
            for (uint64_t v = (uint64_t)src + 1; v <= v_num; v++) offsets[v] = m;
        nbr[i] = dst;
        const uint64_t key = src < dst ? ((uint64_t)src << 32) | dst : ((uint64_t)dst << 32) | src;
        data[i] = dg::edge_data(key, data_seed, weighted);
    }
}

__global__ void row_degrees(const uint64_t *offsets, uint32_t v_num, uint32_t *deg) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < v_num; v += gridDim.x * blockDim.x)
        deg[v] = (uint32_t)(offsets[v + 1] - offsets[v]);
}

}  // namespace

// The undirected CSR of a device edge list (graph.hpp:671-686 doubling): every
// pair contributes both directions, rows are sorted by neighbour, thresholds as
// for a loaded graph.  Built entirely on the device.
extern "C" int dg_graph_create_from_device_edges(const dg_edges *e, dg_graph **out) {
    DG_CHECK(e && out, DG_ERR_ARG, "dg_graph_create_from_device_edges: NULL argument");
    *out = nullptr;
    const uint32_t v_num = e->v_num;
    const uint64_t m = 2 * e->n;
    dg::DeviceGuard guard(e->device);
    std::unique_ptr<dg_graph> g(new dg_graph());
    g->device = e->device;
    g->v_num = v_num;
    g->m = m;
    DG_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    cudaStream_t s = g->stream;
    DG_CUDA(cudaStreamSynchronize(e->stream));
    const unsigned grid = (unsigned)dg::sm_count(e->device) * 8;
    DG_CUDA(g->offsets.alloc((size_t)v_num + 1));
    DG_CUDA(g->out_deg.alloc(v_num));
    DG_CUDA(g->in_deg.alloc(v_num));
    DG_CUDA(g->freq.alloc(v_num));
    DG_CUDA(cudaMemsetAsync(g->freq.p, 0, (size_t)v_num * 4, s));
    if (m == 0) {
        DG_CUDA(cudaMemsetAsync(g->offsets.p, 0, ((size_t)v_num + 1) * 8, s));
        DG_CUDA(cudaMemsetAsync(g->out_deg.p, 0, (size_t)v_num * 4, s));
        DG_CUDA(cudaMemsetAsync(g->in_deg.p, 0, (size_t)v_num * 4, s));
        DG_CUDA(cudaStreamSynchronize(s));
        *out = g.release();
        return DG_OK;
    }
    dg::DevArray<uint64_t> d, alt;
    DG_CUDA(d.alloc(m));
    DG_CUDA(alt.alloc(m));
    double_keys<<<grid, 256, 0, s>>>(e->keys.p, e->n, d.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    cub::DoubleBuffer<uint64_t> db(d.p, alt.p);
    {
        size_t bytes = 0;
        DG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, db, m, 0, 64, s));
        dg::DevArray<uint8_t> tmp;
        DG_CUDA(tmp.alloc(bytes ? bytes : 1));
        DG_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, bytes, db, m, 0, 64, s));
    }
    if (db.Current() != d.p) d.swap(alt);
    alt.release();
    dg::DevArray<uint32_t> nbr;
    dg::DevArray<float> data;
    DG_CUDA(nbr.alloc(m));
    DG_CUDA(data.alloc(m));
    csr_columns<<<grid, 256, 0, s>>>(d.p, m, v_num, e->data_seed, e->weighted, g->offsets.p, nbr.p, data.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaStreamSynchronize(s));
    d.release();
    row_degrees<<<grid, 256, 0, s>>>(g->offsets.p, v_num, g->out_deg.p);
    dg::note_launch();
    DG_CUDA(cudaMemcpyAsync(g->in_deg.p, g->out_deg.p, (size_t)v_num * 4, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(g->entries.alloc(m));
    dg::EventTimer t;
    t.start(s);
    threshold_kernel<<<grid, 256, 0, s>>>(g->offsets.p, nbr.p, data.p, g->out_deg.p, v_num, g->entries.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    t.stop(s);
    DG_CUDA(cudaStreamSynchronize(s));
    g->threshold_ms = t.ms();
    *out = g.release();
    return DG_OK;
}

extern "C" int dg_graph_create(const char *edge_path, uint32_t v_num, int undirected, int device, dg_graph **out) {
    DG_CHECK(edge_path != nullptr, DG_ERR_ARG, "dg_graph_create: path is NULL");
    FILE *f = fopen(edge_path, "rb");
    DG_CHECK(f != nullptr, DG_ERR_IO, "cannot open %s: %s", edge_path, strerror(errno));
    fseek(f, 0, SEEK_END);
    long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size < 0 || size % (long long)sizeof(HostEdge) != 0) {
        fclose(f);
        return dg::fail(DG_ERR_IO, "%s: size %lld is not a multiple of 12-byte edge records", edge_path, size);
    }
    uint64_t n = (uint64_t)size / sizeof(HostEdge);
    std::vector<HostEdge> edges(n ? n : 1);
    size_t got = n ? fread(edges.data(), sizeof(HostEdge), n, f) : 0;
    fclose(f);
    DG_CHECK(got == n, DG_ERR_IO, "%s: short read (%zu of %llu records)", edge_path, got, (unsigned long long)n);
    return build_graph(edges.data(), n, v_num, undirected, device, out);
}

extern "C" void dg_graph_free(dg_graph *g) { delete g; }

extern "C" int dg_graph_get_info(const dg_graph *g, dg_graph_info *info) {
    DG_CHECK(g && info, DG_ERR_ARG, "dg_graph_get_info: NULL argument");
    info->v_num = g->v_num;
    info->m = g->m;
    info->device_bytes = g->offsets.bytes() + g->entries.bytes() + g->out_deg.bytes() + g->in_deg.bytes() +
                         g->freq.bytes() + g->etable.bytes();
    info->threshold_ms = g->threshold_ms;
    return DG_OK;
}

namespace {
__global__ void split_entries(const uint2 *entries, uint64_t m, uint32_t *nbr, uint32_t *thr) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        uint2 e = entries[i];
        if (nbr) nbr[i] = e.x;
        if (thr) thr[i] = e.y;
    }
}
}  // namespace

extern "C" int dg_graph_copy_csr(const dg_graph *g, uint64_t *offsets, uint32_t *neighbours, uint32_t *thresholds,
                                 uint32_t *out_degree, uint32_t *in_degree) {
    DG_CHECK(g, DG_ERR_ARG, "dg_graph_copy_csr: NULL graph");
    dg::DeviceGuard guard(g->device);
    if (offsets) DG_CUDA(cudaMemcpy(offsets, g->offsets.p, ((size_t)g->v_num + 1) * 8, cudaMemcpyDeviceToHost));
    if (out_degree) DG_CUDA(cudaMemcpy(out_degree, g->out_deg.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToHost));
    if (in_degree) DG_CUDA(cudaMemcpy(in_degree, g->in_deg.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToHost));
    if ((neighbours || thresholds) && g->m) {
        dg::DevArray<uint32_t> a, b;
        if (neighbours) DG_CUDA(a.alloc(g->m));
        if (thresholds) DG_CUDA(b.alloc(g->m));
        split_entries<<<dg::sm_count(g->device) * 4, 256, 0, g->stream>>>(g->entries.p, g->m, a.p, b.p); dg::note_launch();
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaStreamSynchronize(g->stream));
        if (neighbours) DG_CUDA(cudaMemcpy(neighbours, a.p, g->m * 4, cudaMemcpyDeviceToHost));
        if (thresholds) DG_CUDA(cudaMemcpy(thresholds, b.p, g->m * 4, cudaMemcpyDeviceToHost));
    }
    return DG_OK;
}

extern "C" int dg_graph_copy_visits(const dg_graph *g, uint32_t *freq) {
    DG_CHECK(g && freq, DG_ERR_ARG, "dg_graph_copy_visits: NULL argument");
    dg::DeviceGuard guard(g->device);
    DG_CUDA(cudaStreamSynchronize(g->stream));
    DG_CUDA(cudaMemcpy(freq, g->freq.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToHost));
    return DG_OK;
}
