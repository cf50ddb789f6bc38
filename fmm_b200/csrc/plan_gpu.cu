// The point stages of the plan build on the device (fmmgpu_fmm_build's plan; the
// reference builds its octree on the host, octree/src/octree/implementation.rs:682,1014,
// and its point order in fmm-exec/src/fmm.rs:36-93):
//   1. the level-16 Morton key of every source and every target (morton.rs:255-272), with
//      the host's arithmetic operation for operation (a subtraction, a division and a
//      multiplication in f64, then the truncation), so the keys are the host's bit for bit;
//   2. the keys of sources ++ targets sorted and made distinct (route_keys on one rank);
//   3. once the host has refined and balanced the tree on those keys, each point's leaf
//      (the last leaf whose first level-16 key is at most the point's key: Morton order
//      partitions the key space) and the stable order of the points by leaf (points of a
//      leaf in caller order), with each leaf's first position and each point's position.
// Sorting is CUB's radix sort (stable), selection CUB's unique.  Build-time work: the
// buffers are allocated per build and freed before it returns.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "morton.hpp"
#include "plan.hpp"

namespace fmmb {

namespace {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("device plan build: ") + what + ": " + cudaGetErrorString(e));
}

template <class V>
struct Buf {
    V* p = nullptr;
    size_t n = 0;
    explicit Buf(size_t count) : n(count) { check(cudaMalloc(&p, sizeof(V) * (count ? count : 1)), "cudaMalloc"); }
    ~Buf() {
        if (p) cudaFree(p);
    }
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
};

struct Box6 {
    double v[6];
};

__global__ void point_keys_kernel(const double* __restrict__ pts, int64_t n, Box6 box, uint64_t* __restrict__ keys) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t size16 = 1u << kDeepest;
    uint32_t id[3];
    for (int k = 0; k < 3; ++k) {
        const double ref = __ddiv_rn(__dsub_rn(pts[3 * i + k], box.v[k]), __dsub_rn(box.v[k + 3], box.v[k]));
        const double s = __dmul_rn(ref, (double)size16);
        const uint64_t c = s <= 0.0 ? 0 : (uint64_t)s;
        id[k] = (uint32_t)(c < (uint64_t)(size16 - 1) ? c : (uint64_t)(size16 - 1));
    }
    keys[i] = morton_encode_hd(id[0], id[1], id[2], kDeepest);
}

// the leaf of each point: upper_bound over the sorted first keys, minus one
__global__ void point_leaf_kernel(const uint64_t* __restrict__ keys, int64_t n, const uint64_t* __restrict__ firsts,
                                  int64_t nfirst, const int32_t* __restrict__ leaf_index, uint32_t* __restrict__ lf,
                                  int64_t* __restrict__ iota) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = keys[i];
    int64_t lo = 0, hi = nfirst;  // first position with firsts[pos] > k
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (firsts[mid] <= k) lo = mid + 1;
        else hi = mid;
    }
    lf[i] = (uint32_t)leaf_index[lo - 1];
    iota[i] = i;
}

// start[j] = the first sorted position whose leaf is >= j (j = 0..nl)
__global__ void leaf_start_kernel(const uint32_t* __restrict__ sorted_lf, int64_t n, int64_t nl,
                                  int64_t* __restrict__ start) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j > nl) return;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)sorted_lf[mid] < j) lo = mid + 1;
        else hi = mid;
    }
    start[j] = lo;
}

__global__ void inverse_kernel(const int64_t* __restrict__ perm, int64_t n, int64_t* __restrict__ pos_of) {
    const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a < n) pos_of[perm[a]] = a;
}

unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

class DevicePointSort final : public PointSort {
   public:
    DevicePointSort(size_t ns, const double* src, size_t nt, const double* tgt, const double box6[6])
        : ns_(ns), nt_(nt), keys_(ns + nt) {
        Box6 b;
        for (int k = 0; k < 6; ++k) b.v[k] = box6[k];
        for (int s = 0; s < 2; ++s) {
            const size_t n = s ? nt : ns;
            if (!n) continue;
            Buf<double> pts(3 * n);
            check(cudaMemcpy(pts.p, s ? tgt : src, sizeof(double) * 3 * n, cudaMemcpyHostToDevice), "copy points");
            point_keys_kernel<<<blocks((int64_t)n), 256>>>(pts.p, (int64_t)n, b, keys_.p + (s ? ns : 0));
            check(cudaGetLastError(), "point keys");
        }
        check(cudaDeviceSynchronize(), "point keys");
    }

    std::vector<uint64_t> distinct_keys() override {
        const size_t n = ns_ + nt_;
        Buf<uint64_t> sorted(n), uniq(n);
        Buf<int64_t> count(1);
        size_t tb = 0, tb2 = 0;
        check(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys_.p, sorted.p, (int64_t)n), "sort size");
        check(cub::DeviceSelect::Unique(nullptr, tb2, sorted.p, uniq.p, count.p, (int64_t)n), "unique size");
        Buf<unsigned char> temp(tb > tb2 ? tb : tb2);
        check(cub::DeviceRadixSort::SortKeys(temp.p, tb, keys_.p, sorted.p, (int64_t)n), "sort");
        check(cub::DeviceSelect::Unique(temp.p, tb2, sorted.p, uniq.p, count.p, (int64_t)n), "unique");
        int64_t nu = 0;
        check(cudaMemcpy(&nu, count.p, sizeof(nu), cudaMemcpyDeviceToHost), "unique count");
        std::vector<uint64_t> out((size_t)nu);
        check(cudaMemcpy(out.data(), uniq.p, sizeof(uint64_t) * (size_t)nu, cudaMemcpyDeviceToHost), "unique keys");
        return out;
    }

    void leaf_order(const std::vector<uint64_t>& firsts, const std::vector<int32_t>& leaf_index, size_t nl,
                    Plan& P) override {
        Buf<uint64_t> df(firsts.size());
        Buf<int32_t> dl(leaf_index.size());
        check(cudaMemcpy(df.p, firsts.data(), sizeof(uint64_t) * firsts.size(), cudaMemcpyHostToDevice), "firsts");
        check(cudaMemcpy(dl.p, leaf_index.data(), sizeof(int32_t) * leaf_index.size(), cudaMemcpyHostToDevice),
              "leaf index");
        for (int s = 0; s < 2; ++s) {
            const size_t n = s ? nt_ : ns_;
            std::vector<int64_t> start(nl + 1, 0), perm(n), pos_of(n);
            if (n) {
                Buf<uint32_t> lf(n), lf_sorted(n);
                Buf<int64_t> iota(n), dperm(n), dstart(nl + 1), dpos(n);
                point_leaf_kernel<<<blocks((int64_t)n), 256>>>(keys_.p + (s ? ns_ : 0), (int64_t)n, df.p,
                                                               (int64_t)firsts.size(), dl.p, lf.p, iota.p);
                check(cudaGetLastError(), "point leaves");
                size_t tb = 0;
                check(cub::DeviceRadixSort::SortPairs(nullptr, tb, lf.p, lf_sorted.p, iota.p, dperm.p, (int64_t)n),
                      "order size");
                Buf<unsigned char> temp(tb);
                check(cub::DeviceRadixSort::SortPairs(temp.p, tb, lf.p, lf_sorted.p, iota.p, dperm.p, (int64_t)n),
                      "order");
                leaf_start_kernel<<<blocks((int64_t)nl + 1), 256>>>(lf_sorted.p, (int64_t)n, (int64_t)nl, dstart.p);
                inverse_kernel<<<blocks((int64_t)n), 256>>>(dperm.p, (int64_t)n, dpos.p);
                check(cudaGetLastError(), "leaf starts");
                check(cudaMemcpy(start.data(), dstart.p, sizeof(int64_t) * (nl + 1), cudaMemcpyDeviceToHost), "starts");
                check(cudaMemcpy(perm.data(), dperm.p, sizeof(int64_t) * n, cudaMemcpyDeviceToHost), "order");
                check(cudaMemcpy(pos_of.data(), dpos.p, sizeof(int64_t) * n, cudaMemcpyDeviceToHost), "positions");
            }
            if (s) {
                P.tgt_start.swap(start);
                P.tgt_perm.swap(perm);
                P.tgt_pos_of.swap(pos_of);
            } else {
                P.src_start.swap(start);
                P.src_perm.swap(perm);
                P.src_pos_of.swap(pos_of);
            }
        }
    }

   private:
    size_t ns_, nt_;
    Buf<uint64_t> keys_;
};

__global__ void pair_keys_kernel(const int64_t* __restrict__ t, const int64_t* __restrict__ s, int64_t n,
                                 uint64_t* __restrict__ keys) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) keys[i] = ((uint64_t)t[i] << 32) | (uint64_t)s[i];
}

__global__ void pair_unpack_kernel(const uint64_t* __restrict__ keys, int64_t n, int64_t* __restrict__ src) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) src[i] = (int64_t)(keys[i] & 0xFFFFFFFFull);
}

// row[t] = the first sorted pair whose target is >= t (t = 0..ntgt)
__global__ void pair_rows_kernel(const uint64_t* __restrict__ keys, int64_t n, int64_t ntgt, int64_t* __restrict__ row) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t > ntgt) return;
    const uint64_t k = (uint64_t)t << 32;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    row[t] = lo;
}

}  // namespace

void sort_close_pairs(int64_t n, const int64_t* t, const int64_t* s, const int32_t* l, int64_t ntgt, int64_t* row,
                      int64_t* src, int32_t* leaf) {
    if (ntgt >= ((int64_t)1 << 31)) throw std::runtime_error("device plan build: too many targets");
    if (n > 0) {
        Buf<uint64_t> keys(n), sorted(n);
        pair_keys_kernel<<<blocks(n), 256>>>(t, s, n, keys.p);
        check(cudaGetLastError(), "pair keys");
        size_t tb = 0;
        check(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, sorted.p, l, leaf, n), "pair sort size");
        Buf<unsigned char> temp(tb);
        check(cub::DeviceRadixSort::SortPairs(temp.p, tb, keys.p, sorted.p, l, leaf, n), "pair sort");
        pair_unpack_kernel<<<blocks(n), 256>>>(sorted.p, n, src);
        pair_rows_kernel<<<blocks(ntgt + 1), 256>>>(sorted.p, n, ntgt, row);
        check(cudaGetLastError(), "pair rows");
        check(cudaDeviceSynchronize(), "pair sort");
    } else {
        check(cudaMemset(row, 0, sizeof(int64_t) * (size_t)(ntgt + 1)), "pair rows");
    }
}

std::unique_ptr<PointSort> device_point_sort(size_t ns, const double* src, size_t nt, const double* tgt,
                                             const double box6[6]) {
    return std::make_unique<DevicePointSort>(ns, src, nt, tgt, box6);
}

}  // namespace fmmb
