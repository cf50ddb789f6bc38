// The evaluator's host-side interface, shared by the C ABI (evaluator.cu) and the
// per-order translation units (evaluator_order.cu, one per compiled expansion order):
// errors, device buffers, per-kind timing, the abstract evaluator and its factory.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fmm_b200.h"
#include "plan.hpp"

namespace fmmb {

// The message fmmgpu_last_error returns on this thread (defined in evaluator.cu).
void set_last_error(const std::string& message);


struct Failure : std::runtime_error {
    int status;
    Failure(int s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

#define CUDA_TRY(expr)                                                                          \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess)                                                                  \
            throw Failure(_e == cudaErrorMemoryAllocation ? FMMGPU_DEVICE_MEMORY : FMMGPU_DEVICE_ERROR, \
                          std::string(#expr) + ": " + cudaGetErrorString(_e));                  \
    } while (0)

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (ptr) cudaFree(ptr);
    }
    void alloc(size_t n) {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = n;
        if (n) CUDA_TRY(cudaMalloc(&ptr, n));
    }
    template <class V>
    void upload(const std::vector<V>& v) {
        alloc(v.size() * sizeof(V) + sizeof(V));
        if (!v.empty()) CUDA_TRY(cudaMemcpy(ptr, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice));
    }
    template <class V>
    V* as() const {
        return static_cast<V*>(ptr);
    }
};

inline int round32(int x) { return (x + 31) / 32 * 32; }


// Per-kind device timing (the reference's KindTiming, fmm-exec/src/fmm.rs:150-153): when
// enabled, every launch is bracketed by two events on the stream and the elapsed times
// are summed per kind after the evaluation.
enum Kind { kLoad = 0, kP2M, kM2M, kL2L, kM2L, kP2L, kFar, kP2P, kKinds };

struct KindTimer {
    bool on = false;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> events;
    std::vector<int> kinds;
    size_t used = 0;
    double ms[kKinds] = {0};
    ~KindTimer() {
        for (auto e : events) cudaEventDestroy(e);
    }
    void begin() {
        used = 0;
        kinds.clear();
    }
    template <class F>
    void run(int kind, F&& launch) {
        if (!on) {
            launch();
            return;
        }
        while (events.size() < used + 2) {
            cudaEvent_t e;
            CUDA_TRY(cudaEventCreate(&e));
            events.push_back(e);
        }
        CUDA_TRY(cudaEventRecord(events[used], stream));
        launch();
        CUDA_TRY(cudaEventRecord(events[used + 1], stream));
        kinds.push_back(kind);
        used += 2;
    }
    void collect() {
        for (int k = 0; k < kKinds; ++k) ms[k] = 0.0;
        if (!on) return;
        CUDA_TRY(cudaStreamSynchronize(stream));
        for (size_t i = 0; i < kinds.size(); ++i) {
            float t = 0.0f;
            CUDA_TRY(cudaEventElapsedTime(&t, events[2 * i], events[2 * i + 1]));
            ms[kinds[i]] += t;
        }
    }
};

// ----------------------------------------------------------------------------------
// The evaluator of one precision T and one degree P.
// ----------------------------------------------------------------------------------
struct EvaluatorBase {
    KindTimer timer;
    // M2L: 1 tensor-core products then the reduce (mixed, p <= 8: the default there),
    // 2 tensor cores fused with the local reduce (an option), 0 SIMT products then the reduce
    int m2l_path = 0;
    virtual int device_status() { return 0; }
    // the device word device_status() reads (nullptr: none), for a copy queued on the
    // evaluator's stream instead of a synchronous read after it
    virtual const int* device_status_word() const { return nullptr; }
    int64_t close_pairs = 0;  // near-singular pairs the mixed form evaluates in f64
    int kinds = 3;  // bit 0 near field (P2P), bit 1 far field; a test hook, 3 in use
    int64_t launches = 0;  // kernels launched by the last evaluation
    int qstride = 1;       // charges per point in the caller's array (all vectors)
    bool first_pass = true;  // vectors run in passes: the first one resets timing and counts
    bool overlap = false;  // near field on its own stream beside the far field (measured: no gain)
    // launch shapes the autotuner may change: warps a block of the mixed P2P kernel
    // (1, 2 or 4) and threads a block of the L2P / M2P kernel (32, 64 or 128)
    int p2p_warps = 4;  // the static block, kX2Warps of p2p_x2.cuh (checked there)
    int leaf_block = 64;
    // the tensor-core M2L tile: 0 the default columns, 1 the alternative (tc_alt_columns)
    int m2l_tile = 0;
    virtual int m2l_tile_columns(int tile) const = 0;
    // mixed P2P: 1 the sources from the near rows' streams mapped at build time (the
    // default when the streams fit), 0 mapped per flush; the same floats
    int p2p_path = 0;
    int64_t p2p_stream_bytes = 0;
    unsigned counted(unsigned grid) {  // wraps the grid of every evaluation launch
        ++launches;
        return grid;
    }
    virtual ~EvaluatorBase() = default;
    virtual void evaluate(const double* d_charges, double* d_phi, double* d_grad) = 0;
    virtual void op_begin(const double* d_charges) = 0;
    virtual void op_level(int kind, int level) = 0;
    virtual void op_output(double* d_phi, double* d_grad) = 0;
    virtual void helmholtz_near(double kre, double kim, const double* d_q, double* d_phi, double* d_grad) = 0;
    // the whole Helmholtz FMM for a real wavenumber (near and far field), device buffers:
    // complex charges [i][v] (qstride vectors a point), outputs [v][i] and [v][i][3] complex
    virtual void helmholtz_fmm(double kre, double kim, const double* d_q, double* d_phi, double* d_grad) = 0;
    // host seconds spent building (or loading) the Helmholtz tables of the last new wavenumber
    double hh_table_seconds = 0.0;
    // the table cache directory of the build ("" none): the Helmholtz tables of each level
    // are loaded from it, or built and stored there
    std::string table_cache_dir;
    virtual void autotune(const double* d_charges, double* d_phi, double* d_grad) = 0;
    virtual void set_m2l_path(int path) = 0;
    virtual void set_p2p_path(int path) = 0;
    virtual int64_t product_chunks() const = 0;
};

// The expansion orders compiled in: each one is its own translation unit
// (evaluator_order.cu built with -DFMMB_P=p), so the orders compile in parallel.
#define FMMB_FOR_EACH_ORDER(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)
constexpr int kMinOrder = 3, kMaxOrder = 12;

// What an evaluator is built from: the plan, the f64 tables (316 M2L, 8 M2M, 8 L2L), the
// stream, the vectors of a pass, gradients, the leaf-scaled coordinates, the M2L form and
// the product budget (0: every M2L product at once).
struct EvaluatorArgs {
    const Plan& plan;
    const std::vector<double>& m2l;
    const std::vector<double>& m2m;
    const std::vector<double>& l2l;
    cudaStream_t stream;
    int m;
    bool gradients;
    const std::vector<double>& us;
    const std::vector<double>& ut;
    bool fused;
    int64_t ybudget;
};

// The evaluator of order P in f64 (mixed = false) or the mixed form; *bytes receives the
// device memory it holds.  Explicitly instantiated once per compiled order.
template <int P>
std::unique_ptr<EvaluatorBase> make_evaluator_at(bool mixed, const EvaluatorArgs& args, size_t* bytes);

}  // namespace fmmb
