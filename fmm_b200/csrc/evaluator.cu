// The C ABI of include/fmm_b200.h: builds (plan on the host, evaluator on the device),
// evaluations (direct launches or one CUDA graph of the whole sweep), the level calls,
// the vector-Jacobian product and the Helmholtz near field.  The evaluator itself is
// evaluator_impl.cuh, compiled once per expansion order (evaluator_order.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fmm_b200.h"
#include "evaluator_base.hpp"
#include "m2l_fused.cuh"
#include "m2l_tc.cuh"
#include "plan.hpp"

namespace fmmb {

namespace {

thread_local std::string g_last_error;

}  // namespace

// The message fmmgpu_last_error returns on this thread (also set by direct.cu).
void set_last_error(const std::string& message) { g_last_error = message; }

std::unique_ptr<EvaluatorBase> make_evaluator(int p, bool mixed, const EvaluatorArgs& args, size_t* bytes) {
#define FMMB_CASE(PP) \
    case PP: return make_evaluator_at<PP>(mixed, args, bytes);
    switch (p) {
        FMMB_FOR_EACH_ORDER(FMMB_CASE)
        default:
            throw Failure(FMMGPU_UNSUPPORTED, "expansion order " + std::to_string(p) + " is not compiled in (" +
                                                  std::to_string(kMinOrder) + " to " + std::to_string(kMaxOrder) + ")");
    }
#undef FMMB_CASE
}

}  // namespace fmmb

// ----------------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------------
using namespace fmmb;

struct fmmgpu_fmm {
    fmmgpu_settings settings;
    Plan plan;
    std::vector<double> m2l, m2m, l2l;
    cudaStream_t stream = nullptr;
    std::unique_ptr<EvaluatorBase> eval;
    DevBuf d_charges, d_phi, d_grad;
    size_t device_bytes = 0;
    int64_t near_pairs = 0;
    bool op_begun = false;  // a level-call evaluation has begun
    int mpass = 1;          // charge vectors per evaluator pass (all of them unless memory says no)
    bool fused = false;     // M2L fused with the local reduce on the tensor cores (mixed, p <= 8)
    int64_t ybudget = 0;    // product buffer bytes of the chunked product path (0: not chunked)
    // whole-evaluation CUDA graph: captured once per (charges, potential, gradient)
    // buffer triple, replayed while the triple and the settings stay the same
    bool graph_on = false;
    cudaGraphExec_t graph = nullptr;
    const void* graph_key[3] = {nullptr, nullptr, nullptr};
    int64_t graph_launches = 0;
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    // vector-Jacobian products: built with targets == sources, the transpose problem is
    // this FMM; otherwise the points are kept and the swapped FMM is built at the first VJP
    bool symmetric = false;
    std::vector<double> src_pts, tgt_pts;
    fmmgpu_fmm* transpose = nullptr;
    DevBuf d_vjp_w, d_vjp_tq, d_vjp_dq, d_vjp_dxs, d_vjp_dxt;
    // the stored forward pass (fmmgpu_fmm_set_vjp_store): the charges and target gradients
    // of the last evaluation, which a VJP with the same charges uses instead of its own
    // forward FMM; off, every VJP recomputes it
    bool vjp_store = false, keep_valid = false;
    DevBuf d_keep_q, d_keep_g, d_keep_flag;
    int64_t vjp_forward_reused = 0;
    DevBuf d_hq, d_hphi, d_hg;  // the Helmholtz host call's device buffers
    DevBuf d_q32, d_out32;      // the f32 host call's charges and (potential, gradient) in f32
    int* h_status = nullptr;    // pinned: the device status word, copied on the stream by the host calls
    int64_t tables_loaded = 0;  // tables taken from the table cache (bits: M2L, M2M, L2L)
    std::string table_cache_dir, tuning_cache_dir;  // the settings' cache directories ("" none)
    bool uploaded = false;         // the plan came from the caller (fmmgpu_upload_plan)
    std::vector<uint8_t> is_leaf;  // per box, for fmmgpu_fmm_plan_arrays
    int64_t tuning_loaded = 0;  // launch shapes taken from the tuning cache
};

namespace fmmb {

// flag = 1 when a[0..n) and b[0..n) differ in any bit (flag starts at 0)
__global__ void differ_kernel(int64_t n, const unsigned long long* __restrict__ a,
                              const unsigned long long* __restrict__ b, int* __restrict__ flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (a[i] != b[i]) {
            *flag = 1;
            return;
        }
}

// the f32 host call's conversions: charges widened to f64 exactly; potentials and
// gradients rounded to the nearest f32 (ties to even)
__global__ void widen_kernel(int64_t n, const float* __restrict__ a, double* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}
__global__ void narrow_kernel(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = __double2float_rn(a[i]);
}
static unsigned grid_of(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }
// potentials [0, np) then gradients [np, np + ng) rounded to f32 in one launch
__global__ void narrow2_kernel(int64_t np, int64_t ng, const double* __restrict__ a, const double* __restrict__ g,
                               float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np + ng; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __double2float_rn(i < np ? a[i] : g[i - np]);
}

// ---- vector-Jacobian products of phi(q, sources, targets) for a cotangent w on phi ----
// dx_t[i] = sum_v w[v][i] grad phi_v(t_i)   (w, phi in the output layout [v][nt])
__global__ void vjp_target_kernel(int64_t nt, int m, const double* __restrict__ w, const double* __restrict__ g,
                                  double* __restrict__ dxt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nt) return;
    double a[3] = {0.0, 0.0, 0.0};
    for (int v = 0; v < m; ++v) {
        const double wv = w[(int64_t)v * nt + i];
        for (int k = 0; k < 3; ++k) a[k] += wv * g[((int64_t)v * nt + i) * 3 + k];
    }
    for (int k = 0; k < 3; ++k) dxt[3 * i + k] = a[k];
}

// [v][n] -> [i][v] (outputs of one FMM as the charges of the transpose one)
__global__ void vjp_transpose_kernel(int64_t n, int m, const double* __restrict__ in, double* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int v = 0; v < m; ++v) out[i * m + v] = in[(int64_t)v * n + i];
}

// dq[j][v] = psi_v(s_j) and dx_s[j] = sum_v q[j][v] grad psi_v(s_j), psi the transpose FMM's
// potentials (charges w at the targets, evaluated at the sources)
__global__ void vjp_source_kernel(int64_t ns, int m, const double* __restrict__ q, const double* __restrict__ psi,
                                  const double* __restrict__ gpsi, double* __restrict__ dq, double* __restrict__ dxs) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= ns) return;
    double a[3] = {0.0, 0.0, 0.0};
    for (int v = 0; v < m; ++v) {
        dq[j * m + v] = psi[(int64_t)v * ns + j];
        const double qv = q[j * m + v];
        for (int k = 0; k < 3; ++k) a[k] += qv * gpsi[((int64_t)v * ns + j) * 3 + k];
    }
    for (int k = 0; k < 3; ++k) dxs[3 * j + k] = a[k];
}

}  // namespace fmmb

namespace {

// One evaluation on the handle's stream: replayed from the CUDA graph when graphs are on
// (and per-kind timing is off), else launched directly.
// The evaluation in passes of f->mpass vectors (all of them when they fit on the device).
void run_passes(fmmgpu_fmm* f, const double* q, double* phi, double* grad) {
    EvaluatorBase& ev = *f->eval;
    const int m = f->settings.vectors;
    const int64_t nt = (int64_t)f->plan.tgt_perm.size();
    for (int v0 = 0; v0 < m; v0 += f->mpass) {
        ev.first_pass = v0 == 0;
        ev.evaluate(q + v0, phi + (int64_t)v0 * nt, grad ? grad + 3 * (int64_t)v0 * nt : nullptr);
    }
    ev.first_pass = true;
}

void run_evaluation(fmmgpu_fmm* f, const double* q, double* phi, double* grad) {
    EvaluatorBase& ev = *f->eval;
    if (!f->graph_on || ev.timer.on) {
        run_passes(f, q, phi, grad);
        return;
    }
    if (!f->graph || f->graph_key[0] != q || f->graph_key[1] != phi || f->graph_key[2] != grad) {
        f->drop_graph();
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(f->stream, cudaStreamCaptureModeThreadLocal));
        try {
            run_passes(f, q, phi, grad);
        } catch (...) {
            cudaStreamEndCapture(f->stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        CUDA_TRY(cudaStreamEndCapture(f->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&f->graph, g, 0);
        cudaGraphDestroy(g);
        CUDA_TRY(e);
        f->graph_key[0] = q;
        f->graph_key[1] = phi;
        f->graph_key[2] = grad;
        f->graph_launches = ev.launches;
    }
    CUDA_TRY(cudaGraphLaunch(f->graph, f->stream));
    ev.launches = f->graph_launches;
}

// with the forward pass stored: keep this evaluation's charges and target gradients
void keep_forward(fmmgpu_fmm* f, const double* q, const double* grad) {
    if (!f->vjp_store || !grad) return;
    const size_t m = f->settings.vectors, ns = f->plan.src_perm.size(), nt = f->plan.tgt_perm.size();
    CUDA_TRY(cudaMemcpyAsync(f->d_keep_q.ptr, q, sizeof(double) * m * ns, cudaMemcpyDeviceToDevice, f->stream));
    CUDA_TRY(cudaMemcpyAsync(f->d_keep_g.ptr, grad, sizeof(double) * 3 * m * nt, cudaMemcpyDeviceToDevice, f->stream));
    f->keep_valid = true;
}

}  // namespace

namespace {

template <class F>
int guarded(F&& f) {
    try {
        f();
        return FMMGPU_OK;
    } catch (const Failure& e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return FMMGPU_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return FMMGPU_INVALID_ARGUMENT;
    }
}

}  // namespace

extern "C" {

void fmmgpu_default_settings(fmmgpu_settings* s) {
    s->p = 6;
    s->precision = FMMGPU_PRECISION_F64;
    s->gradients = 0;
    s->vectors = 1;
    s->max_points_per_leaf = 64;
    s->max_level = 16;
    s->device = 0;
    s->vectors_per_pass = 0;
    s->autotune = 0;
    s->product_bytes = 0;
    s->table_cache = nullptr;
    s->tuning_cache = nullptr;
}

namespace {

void check_settings(const fmmgpu_settings* settings) {
    if (!settings) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
    const fmmgpu_settings& s = *settings;
    if (s.p < 0 || s.vectors < 1 || s.max_points_per_leaf < 1 || s.max_level < 0 || s.max_level > 16 ||
        s.vectors_per_pass < 0 || s.autotune < 0 || s.autotune > 1 || s.product_bytes < 0)
        throw Failure(FMMGPU_INVALID_ARGUMENT, "invalid settings");
    if (s.precision != FMMGPU_PRECISION_F64 && s.precision != FMMGPU_PRECISION_MIXED)
        throw Failure(FMMGPU_UNSUPPORTED, "unknown precision");
}

// leaf-scaled coordinates in the plan's leaf order (CONVENTIONS 3.13)
void leaf_scaled(const Plan& P, const double* src, const double* tgt, std::vector<double>& us,
                 std::vector<double>& ut) {
    us.assign(3 * P.src_perm.size(), 0.0);
    ut.assign(3 * P.tgt_perm.size(), 0.0);
    // leaves in chunks on host threads (each point written once: the same coordinates)
    for_chunks(P.nleaves(), stage_threads(P.nleaves()), [&](size_t, size_t j0, size_t j1) {
        for (size_t j = j0; j < j1; ++j) {
            int b = P.leaf_box[j];
            for (int64_t a = P.src_start[j]; a < P.src_start[j + 1]; ++a) {
                int64_t i = P.src_perm[a];
                for (int k = 0; k < 3; ++k)
                    us[3 * a + k] = leaf_coordinate(src[3 * i + k], P.lower[k], P.side, P.level[b], P.idx[3 * b + k]);
            }
            for (int64_t a = P.tgt_start[j]; a < P.tgt_start[j + 1]; ++a) {
                int64_t i = P.tgt_perm[a];
                for (int k = 0; k < 3; ++k)
                    ut[3 * a + k] = leaf_coordinate(tgt[3 * i + k], P.lower[k], P.side, P.level[b], P.idx[3 * b + k]);
            }
        }
    });
}

int64_t count_near_pairs(const Plan& P) {
    int64_t n = 0;
    for (size_t j = 0; j < P.nleaves(); ++j) {
        int64_t nt_j = P.tgt_start[j + 1] - P.tgt_start[j];
        for (int64_t e = P.near.row[j]; e < P.near.row[j + 1]; ++e) {
            int sj = P.near.col[e];
            n += nt_j * (P.src_start[sj + 1] - P.src_start[sj]);
        }
    }
    return n;
}

// The f64 operator tables of degree p: from the table cache when the settings name one
// (a file missing or rejected is rebuilt and stored; a failed store leaves the build as it
// is, as the reference's load_or_build never fails because of its cache), else built.
// The settings' cache directories are copied (the caller's strings need not outlive the
// build) and the handle's copy of the settings keeps no pointer to them.
void keep_cache_dirs(fmmgpu_fmm* f) {
    f->table_cache_dir = f->settings.table_cache ? f->settings.table_cache : "";
    f->tuning_cache_dir = f->settings.tuning_cache ? f->settings.tuning_cache : "";
    f->settings.table_cache = nullptr;
    f->settings.tuning_cache = nullptr;
}

void load_or_build_tables(fmmgpu_fmm* f) {
    const fmmgpu_settings& s = f->settings;
    const std::string& dir = f->table_cache_dir;
    const int p = s.p;
    const size_t n2 = (size_t)(p + 1) * (p + 1) * (p + 1) * (p + 1);
    struct Kind {
        int code;
        size_t sets;
        std::vector<double>* out;
        void (*build)(int, std::vector<double>&);
        int bit;
    } kinds[3] = {{kTableM2l, 316, &f->m2l, build_m2l_tables, 1},
                  {kTableM2m, 8, &f->m2m, build_m2m_tables, 2},
                  {kTableL2l, 8, &f->l2l, build_l2l_tables, 4}};
    f->tables_loaded = 0;
    for (const Kind& k : kinds) {
        std::string why;
        if (!dir.empty() && table_cache_load(dir, k.code, p, 0.0, k.sets * n2, *k.out, &why)) {
            f->tables_loaded |= k.bit;
            continue;
        }
        k.build(p, *k.out);
        if (!dir.empty()) table_cache_store(dir, k.code, p, 0.0, *k.out, &why);
    }
}

// Host part of a build: plan, tables, leaf-scaled coordinates (no device work).
std::unique_ptr<fmmgpu_fmm> build_host(const fmmgpu_settings* settings, size_t ns, const double* src, size_t nt,
                                       const double* tgt, std::vector<double>& us, std::vector<double>& ut,
                                       bool device_points = false) {
    check_settings(settings);
    const fmmgpu_settings& s = *settings;
    if ((ns && !src) || (nt && !tgt)) throw Failure(FMMGPU_INVALID_ARGUMENT, "null points");
    auto f = std::make_unique<fmmgpu_fmm>();
    f->settings = s;
    keep_cache_dirs(f.get());
    if (device_points) CUDA_TRY(cudaSetDevice(s.device));
    f->plan = build_plan(ns, src, nt, tgt, s.max_level, s.max_points_per_leaf, device_points);
    load_or_build_tables(f.get());
    leaf_scaled(f->plan, src, tgt, us, ut);
    f->near_pairs = count_near_pairs(f->plan);
    return f;
}

// Host part of a batch build: every cloud's plan (in parallel over the host's threads),
// merged into one forest; the clouds' points are consecutive in the caller's arrays.
std::unique_ptr<fmmgpu_fmm> build_host_batch(const fmmgpu_settings* settings, size_t ncloud, const size_t* ns,
                                             const double* src, const size_t* nt, const double* tgt,
                                             std::vector<double>& us, std::vector<double>& ut) {
    check_settings(settings);
    const fmmgpu_settings& s = *settings;
    if (ncloud == 0 || !ns) throw Failure(FMMGPU_INVALID_ARGUMENT, "no clouds");
    const bool same = nt == nullptr;  // targets are the sources
    std::vector<TreePart> parts(ncloud);
    int64_t so = 0, to = 0;
    for (size_t c = 0; c < ncloud; ++c) {
        parts[c].src_offset = so;
        parts[c].tgt_offset = to;
        so += (int64_t)ns[c];
        to += (int64_t)(same ? ns[c] : nt[c]);
    }
    if ((so && !src) || (to && !same && !tgt)) throw Failure(FMMGPU_INVALID_ARGUMENT, "null points");
    std::vector<std::string> errors(ncloud);
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t c; (c = next.fetch_add(1)) < ncloud;) {
            try {
                TreePart& tp = parts[c];
                const double* cs = src + 3 * tp.src_offset;
                const double* ct = same ? cs : tgt + 3 * tp.tgt_offset;
                const size_t cnt = same ? ns[c] : nt[c];
                // one host thread a cloud: the clouds already run on all of them
                tp.plan = build_plan(ns[c], cs, cnt, ct, s.max_level, s.max_points_per_leaf, false, 1);
                leaf_scaled(tp.plan, cs, ct, tp.us, tp.ut);
            } catch (const std::exception& e) {
                errors[c] = e.what();
            }
        }
    };
    const unsigned nthreads = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)ncloud));
    std::vector<std::thread> pool;
    for (unsigned i = 1; i < nthreads; ++i) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    for (size_t c = 0; c < ncloud; ++c)
        if (!errors[c].empty()) throw Failure(FMMGPU_INVALID_ARGUMENT, "cloud " + std::to_string(c) + ": " + errors[c]);
    auto f = std::make_unique<fmmgpu_fmm>();
    f->settings = s;
    keep_cache_dirs(f.get());
    f->plan = merge_plans(parts, us, ut);
    load_or_build_tables(f.get());
    f->near_pairs = count_near_pairs(f->plan);
    return f;
}

// Device part of a build: the evaluator (plan upload, tables, buffers) on the device.
void build_device(fmmgpu_fmm* f, const std::vector<double>& us, const std::vector<double>& ut) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw Failure(FMMGPU_NO_DEVICE, "no CUDA device is visible");
    }
    const fmmgpu_settings& s = f->settings;
    CUDA_TRY(cudaSetDevice(s.device));
    const Plan& P = f->plan;
    int least = 0, greatest = 0;  // the far-field chain is the critical path: highest priority
    CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CUDA_TRY(cudaStreamCreateWithPriority(&f->stream, cudaStreamNonBlocking, greatest));
    // the fused M2L is an option (fmmgpu_fmm_set_m2l_path 2), not the default: measured slower
    // than the product path (its scattered f32 reductions into the locals cost more than
    // writing and re-reading the products)
    f->fused = false;
    // vectors per pass: every per-vector buffer (expansions, translation products, partial
    // outputs) for as many vectors as fit in 60% of the free memory.  The M2L products (Y:
    // one row per V pair and vector) are held for every pair at once when they fit beside
    // the rest; otherwise in a buffer of at most 20% of the free memory, filled chunk by
    // chunk (the chunked product path: the same floats)
    {
        const size_t nc = (size_t)(s.p + 1) * (s.p + 1), ys = (nc + 31) / 32 * 32, ms = (nc + 3) / 4 * 4;
        const size_t tsz = s.precision == FMMGPU_PRECISION_F64 ? 8 : 4;
        const size_t nsrc = P.src_perm.size(), ntgt = P.tgt_perm.size();
        const size_t y_vec = f->fused ? 0 : tsz * ys * (P.v.nnz() + 1);
        const size_t per_vec = tsz * (2 * P.nboxes() * ms + P.nboxes() * ys + nsrc) + (tsz == 4 ? 8 * nsrc : 0) +
                               8 * ntgt * (s.gradients ? 4 : 1) * 2 + 8 * ntgt * (s.gradients ? 4 : 1) + 8 * nsrc;
        size_t free_b = 0, total_b = 0;
        CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        const size_t budget = (size_t)(0.6 * (double)free_b);
        const size_t y_all = y_vec * (size_t)s.vectors;
        size_t ycap = 0;  // product buffer bytes when chunked
        size_t fit = (size_t)s.vectors;
        if (s.product_bytes > 0) {
            ycap = (size_t)s.product_bytes;
            fit = budget > ycap && per_vec ? (budget - ycap) / per_vec : 1;
        } else if (per_vec * (size_t)s.vectors + y_all > budget) {
            ycap = std::min(y_all, (size_t)(0.2 * (double)free_b));
            fit = budget > ycap && per_vec ? (budget - ycap) / per_vec : 1;
        }
        int want = (int)std::max<size_t>(1, std::min<size_t>((size_t)s.vectors, fit));
        if (s.vectors_per_pass > 0) want = std::min(s.vectors_per_pass, s.vectors);
        if (f->fused) want = std::min(want, fused_tile_columns(s.p));
        if (s.precision == FMMGPU_PRECISION_MIXED && tc_tile_columns(s.p) > 0)
            want = std::min(want, tc_tile_columns(s.p));
        // every pass holds the same number of vectors (the buffers' and the kernels' m): the
        // largest divisor of the vector count not above the wanted size
        while (s.vectors % want) --want;
        f->mpass = want;
        f->ybudget = (ycap > 0 && y_vec * (size_t)want > ycap) ? (int64_t)ycap : 0;
    }
    size_t bytes = 0;
    const bool mixed = s.precision == FMMGPU_PRECISION_MIXED;
    const EvaluatorArgs args{P, f->m2l, f->m2m, f->l2l, f->stream, f->mpass, s.gradients != 0, us, ut,
                             mixed && f->fused, f->ybudget};
    f->eval = make_evaluator(s.p, mixed, args, &bytes);
    f->eval->qstride = s.vectors;
    const size_t ns = P.src_perm.size(), nt = P.tgt_perm.size();
    f->d_charges.alloc(sizeof(double) * (size_t)s.vectors * (ns + 1));
    f->d_phi.alloc(sizeof(double) * (size_t)s.vectors * (nt + 1));
    if (s.gradients) f->d_grad.alloc(sizeof(double) * 3 * (size_t)s.vectors * (nt + 1));
    f->device_bytes = bytes + f->d_charges.bytes + f->d_phi.bytes + f->d_grad.bytes;
    f->eval->table_cache_dir = f->table_cache_dir;
    if (s.autotune) {
        // a choice kept in the tuning cache for this device, precision, p and gradients
        // setting is used as it is; otherwise the shapes are timed and the choice stored
        TuningKey key;
        std::map<std::string, int> entries;
        const std::string g = s.gradients ? "gradients:" : "potentials:";
        bool cached = false;
        if (!f->tuning_cache_dir.empty()) {
            cudaDeviceProp prop{};
            CUDA_TRY(cudaGetDeviceProperties(&prop, s.device));
            key.device = std::string(prop.name) + " sm_" + std::to_string(prop.major) + std::to_string(prop.minor) +
                         " " + std::to_string(prop.multiProcessorCount) + " SMs";
            key.compiler = "nvcc cudart " + std::to_string(CUDART_VERSION) + " sm_100a";
            key.precision = s.precision == FMMGPU_PRECISION_F64 ? "f64" : "mixed";
            key.p = s.p;
            std::string why;
            if (tuning_cache_load(f->tuning_cache_dir, key, entries, &why) && entries.count(g + "p2p_warps") &&
                entries.count(g + "leaf_block")) {
                const int w = entries[g + "p2p_warps"], b = entries[g + "leaf_block"];
                const int t = entries.count(g + "m2l_tile") ? entries[g + "m2l_tile"] : 0;
                if ((w == 1 || w == 2 || w == 4) && (b == 32 || b == 64 || b == 128) && (t == 0 || t == 1)) {
                    f->eval->p2p_warps = w;
                    f->eval->leaf_block = b;
                    f->eval->m2l_tile = t;
                    cached = true;
                }
            }
        }
        if (!cached) {
            // the launch shapes timed on this plan with zero charges: the charges change no
            // branch and no launch, so they time as any others
            CUDA_TRY(cudaMemsetAsync(f->d_charges.ptr, 0, f->d_charges.bytes, f->stream));
            f->eval->autotune(f->d_charges.as<double>(), f->d_phi.as<double>(),
                              s.gradients ? f->d_grad.as<double>() : nullptr);
            if (f->eval->device_status()) throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
            if (!f->tuning_cache_dir.empty()) {
                entries[g + "p2p_warps"] = f->eval->p2p_warps;
                entries[g + "leaf_block"] = f->eval->leaf_block;
                entries[g + "m2l_tile"] = f->eval->m2l_tile;
                std::string why;
                tuning_cache_store(f->tuning_cache_dir, key, entries, &why);
            }
        }
        f->tuning_loaded = cached ? 1 : 0;
    }
    CUDA_TRY(cudaDeviceSynchronize());
}

}  // namespace

int fmmgpu_plan_build(const fmmgpu_settings* settings, size_t ns, const double* src, size_t nt,
                      const double* tgt, fmmgpu_fmm** out) {
    return guarded([&] {
        if (!out) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        std::vector<double> us, ut;
        auto f = build_host(settings, ns, src, nt, tgt, us, ut);
        *out = f.release();
    });
}

namespace {

// Host part of a build on a caller's plan: checks, tables, leaf-scaled coordinates (every
// point inside its leaf, within 2^-20 of the leaf's half-width).
std::unique_ptr<fmmgpu_fmm> build_host_uploaded(const fmmgpu_settings* settings, const fmmgpu_plan_arrays* pa,
                                                size_t ns, const double* src, size_t nt, const double* tgt,
                                                std::vector<double>& us, std::vector<double>& ut) {
    check_settings(settings);
    if (!pa) throw Failure(FMMGPU_INVALID_ARGUMENT, "null plan");
    if ((ns && !src) || (nt && !tgt)) throw Failure(FMMGPU_INVALID_ARGUMENT, "null points");
    for (size_t i = 0; i < 3 * ns; ++i)
        if (!std::isfinite(src[i])) throw Failure(FMMGPU_INVALID_ARGUMENT, "non-finite point coordinate");
    for (size_t i = 0; i < 3 * nt; ++i)
        if (!std::isfinite(tgt[i])) throw Failure(FMMGPU_INVALID_ARGUMENT, "non-finite point coordinate");
    auto f = std::make_unique<fmmgpu_fmm>();
    f->settings = *settings;
    keep_cache_dirs(f.get());
    f->plan = plan_from_arrays(*pa, ns, nt);
    f->uploaded = true;
    load_or_build_tables(f.get());
    leaf_scaled(f->plan, src, tgt, us, ut);
    const double lim = 1.0 + std::ldexp(1.0, -20);
    for (const std::vector<double>* u : {&us, &ut})
        for (size_t i = 0; i < u->size(); ++i)
            if (!(std::fabs((*u)[i]) <= lim))
                throw Failure(FMMGPU_INVALID_ARGUMENT, std::string("uploaded plan: a ") + (u == &us ? "source" : "target") +
                                                           " point lies outside its leaf");
    f->near_pairs = count_near_pairs(f->plan);
    return f;
}

}  // namespace

int fmmgpu_plan_from_arrays(const fmmgpu_settings* settings, const fmmgpu_plan_arrays* plan, size_t ns,
                            const double* src, size_t nt, const double* tgt, fmmgpu_fmm** out) {
    return guarded([&] {
        if (!out) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        std::vector<double> us, ut;
        auto f = build_host_uploaded(settings, plan, ns, src, nt, tgt, us, ut);
        *out = f.release();
    });
}

int fmmgpu_upload_plan(const fmmgpu_settings* settings, const fmmgpu_plan_arrays* plan, size_t ns,
                       const double* src, size_t nt, const double* tgt, fmmgpu_fmm** out) {
    return guarded([&] {
        if (!out) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            throw Failure(FMMGPU_NO_DEVICE, "no CUDA device is visible");
        }
        std::vector<double> us, ut;
        auto f = build_host_uploaded(settings, plan, ns, src, nt, tgt, us, ut);
        build_device(f.get(), us, ut);
        f->symmetric = src == tgt && ns == nt;
        *out = f.release();
    });
}

int fmmgpu_fmm_plan_arrays(const fmmgpu_fmm* f, fmmgpu_plan_arrays* a) {
    return guarded([&] {
        if (!f || !a) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        const Plan& P = f->plan;
        if (!P.box_side.empty()) throw Failure(FMMGPU_UNSUPPORTED, "a multi-cloud forest is not one plan");
        auto* self = const_cast<fmmgpu_fmm*>(f);
        self->is_leaf.assign(P.nboxes(), 0);
        for (size_t j = 0; j < P.nleaves(); ++j) self->is_leaf[P.leaf_box[j]] = 1;
        a->nlevels = P.nlevels;
        a->level_start = P.level_start.data();
        a->keys = P.key.data();
        a->is_leaf = self->is_leaf.data();
        for (int k = 0; k < 3; ++k) a->lower[k] = P.lower[k];
        a->side = P.side;
        a->source_offsets = P.src_start.data();
        a->target_offsets = P.tgt_start.data();
        a->source_order = P.src_perm.data();
        a->target_order = P.tgt_perm.data();
        a->near_rows = P.near.row.data();
        a->near = P.near.col.data();
        a->w_rows = P.w.row.data();
        a->w = P.w.col.data();
        a->x_rows = P.x.row.data();
        a->x = P.x.col.data();
        a->v_rows = P.v.row.data();
        a->v = P.v.col.data();
        a->v_offsets = P.v.aux.data();
    });
}

int fmmgpu_fmm_build(const fmmgpu_settings* settings, size_t ns, const double* src, size_t nt,
                     const double* tgt, fmmgpu_fmm** out) {
    return guarded([&] {
        if (!out) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            throw Failure(FMMGPU_NO_DEVICE, "no CUDA device is visible");
        }
        std::vector<double> us, ut;
        auto f = build_host(settings, ns, src, nt, tgt, us, ut, true);  // the point stages on the GPU
        build_device(f.get(), us, ut);
        f->symmetric = src == tgt && ns == nt;
        if (!f->symmetric) {
            f->src_pts.assign(src, src + 3 * ns);
            f->tgt_pts.assign(tgt, tgt + 3 * nt);
        }
        *out = f.release();
    });
}

int fmmgpu_batch_plan_build(const fmmgpu_settings* settings, size_t ncloud, const size_t* nsources,
                            const double* sources, const size_t* ntargets, const double* targets, fmmgpu_fmm** out) {
    return guarded([&] {
        if (!out) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        std::vector<double> us, ut;
        auto f = build_host_batch(settings, ncloud, nsources, sources, ntargets, targets, us, ut);
        *out = f.release();
    });
}

int fmmgpu_batch_build(const fmmgpu_settings* settings, size_t ncloud, const size_t* nsources, const double* sources,
                       const size_t* ntargets, const double* targets, fmmgpu_fmm** out) {
    return guarded([&] {
        if (!out) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            throw Failure(FMMGPU_NO_DEVICE, "no CUDA device is visible");
        }
        std::vector<double> us, ut;
        auto f = build_host_batch(settings, ncloud, nsources, sources, ntargets, targets, us, ut);
        build_device(f.get(), us, ut);
        *out = f.release();
    });
}

int fmmgpu_fmm_evaluate_device(fmmgpu_fmm* f, const double* charges, double* potential, double* gradient) {
    return guarded([&] {
        if (!f || !charges || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        run_evaluation(f, charges, potential, f->settings.gradients ? gradient : nullptr);
        keep_forward(f, charges, f->settings.gradients ? gradient : nullptr);
    });
}

// The end of a host call: the device status word is copied on the evaluator's stream
// into a pinned word, then one synchronisation covers the copies and the check.
static void finish_host_call(fmmgpu_fmm* f) {
    const int* w = f->eval->device_status_word();
    if (w) {
        if (!f->h_status) CUDA_TRY(cudaMallocHost(&f->h_status, sizeof(int)));
        CUDA_TRY(cudaMemcpyAsync(f->h_status, w, sizeof(int), cudaMemcpyDeviceToHost, f->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(f->stream));
    if (w && *f->h_status) throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
}

int fmmgpu_fmm_evaluate(fmmgpu_fmm* f, const double* charges, double* potential, double* gradient) {
    return guarded([&] {
        if (!f || !charges || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const size_t m = f->settings.vectors;
        const size_t ns = f->plan.src_perm.size(), nt = f->plan.tgt_perm.size();
        CUDA_TRY(cudaMemcpyAsync(f->d_charges.ptr, charges, sizeof(double) * m * ns, cudaMemcpyHostToDevice, f->stream));
        run_evaluation(f, f->d_charges.as<double>(), f->d_phi.as<double>(),
                       f->settings.gradients ? f->d_grad.as<double>() : nullptr);
        keep_forward(f, f->d_charges.as<double>(), f->settings.gradients ? f->d_grad.as<double>() : nullptr);
        CUDA_TRY(cudaMemcpyAsync(potential, f->d_phi.ptr, sizeof(double) * m * nt, cudaMemcpyDeviceToHost, f->stream));
        if (f->settings.gradients)
            CUDA_TRY(cudaMemcpyAsync(gradient, f->d_grad.ptr, sizeof(double) * 3 * m * nt, cudaMemcpyDeviceToHost,
                                     f->stream));
        finish_host_call(f);
    });
}

int fmmgpu_fmm_evaluate_f32(fmmgpu_fmm* f, const float* charges, float* potential, float* gradient) {
    return guarded([&] {
        if (!f || !charges || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const int64_t m = f->settings.vectors;
        const int64_t ns = (int64_t)f->plan.src_perm.size(), nt = (int64_t)f->plan.tgt_perm.size();
        const int64_t nq = m * ns, nout = m * nt * (f->settings.gradients ? 4 : 1);
        if (f->d_q32.bytes < sizeof(float) * (size_t)(nq + 1)) f->d_q32.alloc(sizeof(float) * (size_t)(nq + 1));
        if (f->d_out32.bytes < sizeof(float) * (size_t)(nout + 1)) f->d_out32.alloc(sizeof(float) * (size_t)(nout + 1));
        cudaStream_t s = f->stream;
        if (nq) {
            CUDA_TRY(cudaMemcpyAsync(f->d_q32.ptr, charges, sizeof(float) * nq, cudaMemcpyHostToDevice, s));
            widen_kernel<<<grid_of(nq), 256, 0, s>>>(nq, f->d_q32.as<float>(), f->d_charges.as<double>());
            CUDA_TRY(cudaGetLastError());
        }
        run_evaluation(f, f->d_charges.as<double>(), f->d_phi.as<double>(),
                       f->settings.gradients ? f->d_grad.as<double>() : nullptr);
        keep_forward(f, f->d_charges.as<double>(), f->settings.gradients ? f->d_grad.as<double>() : nullptr);
        const int64_t np = m * nt, ng = f->settings.gradients ? 3 * np : 0;
        if (np) {
            float* o = f->d_out32.as<float>();
            narrow2_kernel<<<grid_of(np + ng), 256, 0, s>>>(np, ng, f->d_phi.as<double>(),
                                                            ng ? f->d_grad.as<double>() : nullptr, o);
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaMemcpyAsync(potential, o, sizeof(float) * np, cudaMemcpyDeviceToHost, s));
            if (ng) CUDA_TRY(cudaMemcpyAsync(gradient, o + np, sizeof(float) * ng, cudaMemcpyDeviceToHost, s));
        }
        finish_host_call(f);
    });
}

int fmmgpu_fmm_vjp(fmmgpu_fmm* f, const double* charges, const double* cotangent, double* dcharges,
                   double* dsources, double* dtargets) {
    return guarded([&] {
        if (!f || !charges || !cotangent || !dcharges || !dsources || !dtargets)
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        if (!f->settings.gradients) throw Failure(FMMGPU_INVALID_ARGUMENT, "a VJP needs an FMM built with gradients");
        if (f->plan.box_side.size()) throw Failure(FMMGPU_UNSUPPORTED, "VJPs of multi-cloud batches are not offered");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const int m = f->settings.vectors;
        const int64_t ns = (int64_t)f->plan.src_perm.size(), nt = (int64_t)f->plan.tgt_perm.size();
        fmmgpu_fmm* T = f;
        if (!f->symmetric && f->uploaded)
            throw Failure(FMMGPU_UNSUPPORTED, "a VJP on an uploaded plan needs targets == sources");
        if (!f->symmetric) {
            if (!f->transpose) {  // the swapped problem: charges at the targets, evaluated at the sources
                std::vector<double> us, ut;
                auto t = build_host(&f->settings, (size_t)nt, f->tgt_pts.data(), (size_t)ns, f->src_pts.data(), us, ut,
                                    true);
                build_device(t.get(), us, ut);
                t->symmetric = true;  // never asked for its own transpose
                f->transpose = t.release();
            }
            T = f->transpose;
        }
        f->d_vjp_w.alloc(sizeof(double) * (size_t)m * (nt + 1));
        f->d_vjp_tq.alloc(sizeof(double) * (size_t)m * (nt + 1));
        f->d_vjp_dq.alloc(sizeof(double) * (size_t)m * (ns + 1));
        f->d_vjp_dxs.alloc(sizeof(double) * 3 * (ns + 1));
        f->d_vjp_dxt.alloc(sizeof(double) * 3 * (nt + 1));
        cudaStream_t s = f->stream;
        CUDA_TRY(cudaMemcpyAsync(f->d_charges.ptr, charges, sizeof(double) * m * ns, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(f->d_vjp_w.ptr, cotangent, sizeof(double) * m * nt, cudaMemcpyHostToDevice, s));
        // forward pass: grad phi at the targets, from the stored forward pass when its
        // charges are these (bit for bit, checked on the device), else recomputed
        bool reuse = false;
        if (f->vjp_store && f->keep_valid) {
            CUDA_TRY(cudaMemsetAsync(f->d_keep_flag.ptr, 0, sizeof(int), s));
            const int64_t n = (int64_t)m * ns;
            if (n)
                differ_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(
                    n, f->d_charges.as<unsigned long long>(), f->d_keep_q.as<unsigned long long>(),
                    f->d_keep_flag.as<int>());
            int differ = 1;
            CUDA_TRY(cudaMemcpyAsync(&differ, f->d_keep_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaStreamSynchronize(s));
            reuse = differ == 0;
        }
        if (reuse) {
            ++f->vjp_forward_reused;
        } else {
            run_evaluation(f, f->d_charges.as<double>(), f->d_phi.as<double>(), f->d_grad.as<double>());
            keep_forward(f, f->d_charges.as<double>(), f->d_grad.as<double>());
        }
        const double* fwd_grad = reuse ? f->d_keep_g.as<double>() : f->d_grad.as<double>();
        const unsigned bt = (unsigned)((nt + 255) / 256), bs = (unsigned)((ns + 255) / 256);
        if (nt) {
            vjp_target_kernel<<<bt, 256, 0, s>>>(nt, m, f->d_vjp_w.as<double>(), fwd_grad,
                                                f->d_vjp_dxt.as<double>());
            vjp_transpose_kernel<<<bt, 256, 0, s>>>(nt, m, f->d_vjp_w.as<double>(), f->d_vjp_tq.as<double>());
        }
        CUDA_TRY(cudaGetLastError());
        // transpose pass: charges w at the targets, potentials and gradients at the sources
        if (T != f) CUDA_TRY(cudaStreamSynchronize(s));  // T runs on its own stream
        run_evaluation(T, f->d_vjp_tq.as<double>(), T->d_phi.as<double>(), T->d_grad.as<double>());
        if (T != f) CUDA_TRY(cudaStreamSynchronize(T->stream));
        if (ns)
            vjp_source_kernel<<<bs, 256, 0, s>>>(ns, m, f->d_charges.as<double>(), T->d_phi.as<double>(),
                                                T->d_grad.as<double>(), f->d_vjp_dq.as<double>(),
                                                f->d_vjp_dxs.as<double>());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(dcharges, f->d_vjp_dq.ptr, sizeof(double) * m * ns, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(dsources, f->d_vjp_dxs.ptr, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(dtargets, f->d_vjp_dxt.ptr, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (f->eval->device_status() || T->eval->device_status())
            throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
    });
}

int fmmgpu_helmholtz_near(fmmgpu_fmm* f, double k_re, double k_im, const double* charges, double* potential,
                          double* gradient) {
    return guarded([&] {
        if (!f || !charges || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        if (!std::isfinite(k_re) || !std::isfinite(k_im))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "the wavenumber must be finite");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const size_t m = f->settings.vectors;
        const size_t ns = f->plan.src_perm.size(), nt = f->plan.tgt_perm.size();
        DevBuf q, phi, g;
        q.alloc(sizeof(double) * 2 * m * (ns + 1));
        phi.alloc(sizeof(double) * 2 * m * (nt + 1));
        if (f->settings.gradients) g.alloc(sizeof(double) * 6 * m * (nt + 1));
        CUDA_TRY(cudaMemcpyAsync(q.ptr, charges, sizeof(double) * 2 * m * ns, cudaMemcpyHostToDevice, f->stream));
        for (int v0 = 0; v0 < (int)m; v0 += f->mpass) {
            f->eval->first_pass = v0 == 0;
            f->eval->helmholtz_near(k_re, k_im, q.as<double>() + 2 * v0, phi.as<double>() + 2 * (size_t)v0 * nt,
                                    f->settings.gradients ? g.as<double>() + 6 * (size_t)v0 * nt : nullptr);
        }
        f->eval->first_pass = true;
        CUDA_TRY(cudaMemcpyAsync(potential, phi.ptr, sizeof(double) * 2 * m * nt, cudaMemcpyDeviceToHost, f->stream));
        if (f->settings.gradients)
            CUDA_TRY(cudaMemcpyAsync(gradient, g.ptr, sizeof(double) * 6 * m * nt, cudaMemcpyDeviceToHost, f->stream));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
    });
}

int fmmgpu_helmholtz_evaluate_device(fmmgpu_fmm* f, double k_re, double k_im, const double* charges,
                                     double* potential, double* gradient) {
    return guarded([&] {
        if (!f || !charges || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        if (!std::isfinite(k_re) || !std::isfinite(k_im))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "the wavenumber must be finite");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const size_t m = f->settings.vectors;
        const size_t nt = f->plan.tgt_perm.size();
        for (int v0 = 0; v0 < (int)m; v0 += f->mpass) {
            f->eval->first_pass = v0 == 0;
            f->eval->helmholtz_fmm(k_re, k_im, charges + 2 * v0, potential + 2 * (size_t)v0 * nt,
                                   f->settings.gradients ? gradient + 6 * (size_t)v0 * nt : nullptr);
        }
        f->eval->first_pass = true;
    });
}

int fmmgpu_helmholtz_evaluate(fmmgpu_fmm* f, double k_re, double k_im, const double* charges, double* potential,
                              double* gradient) {
    return guarded([&] {
        if (!f || !charges || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const size_t m = f->settings.vectors;
        const size_t ns = f->plan.src_perm.size(), nt = f->plan.tgt_perm.size();
        if (f->d_hq.bytes < sizeof(double) * 2 * m * (ns + 1)) {
            f->d_hq.alloc(sizeof(double) * 2 * m * (ns + 1));
            f->d_hphi.alloc(sizeof(double) * 2 * m * (nt + 1));
            if (f->settings.gradients) f->d_hg.alloc(sizeof(double) * 6 * m * (nt + 1));
        }
        CUDA_TRY(cudaMemcpyAsync(f->d_hq.ptr, charges, sizeof(double) * 2 * m * ns, cudaMemcpyHostToDevice,
                                 f->stream));
        const int rc = fmmgpu_helmholtz_evaluate_device(f, k_re, k_im, f->d_hq.as<double>(), f->d_hphi.as<double>(),
                                                        f->settings.gradients ? f->d_hg.as<double>() : nullptr);
        if (rc != FMMGPU_OK) throw Failure(rc, g_last_error);
        CUDA_TRY(cudaMemcpyAsync(potential, f->d_hphi.ptr, sizeof(double) * 2 * m * nt, cudaMemcpyDeviceToHost,
                                 f->stream));
        if (f->settings.gradients)
            CUDA_TRY(cudaMemcpyAsync(gradient, f->d_hg.ptr, sizeof(double) * 6 * m * nt, cudaMemcpyDeviceToHost,
                                     f->stream));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        if (f->eval->device_status()) throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
    });
}

int fmmgpu_helmholtz_evaluate_f32(fmmgpu_fmm* f, double k_re, double k_im, const float* charges, float* potential,
                                  float* gradient) {
    return guarded([&] {
        if (!f || !charges || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const int64_t m = f->settings.vectors;
        const int64_t ns = (int64_t)f->plan.src_perm.size(), nt = (int64_t)f->plan.tgt_perm.size();
        if (f->d_hq.bytes < sizeof(double) * 2 * m * (ns + 1)) {
            f->d_hq.alloc(sizeof(double) * 2 * m * (ns + 1));
            f->d_hphi.alloc(sizeof(double) * 2 * m * (nt + 1));
            if (f->settings.gradients) f->d_hg.alloc(sizeof(double) * 6 * m * (nt + 1));
        }
        // complex numbers as (re, im) pairs: the conversions act on the 2n reals
        const int64_t nq = 2 * m * ns, np = 2 * m * nt, ng = f->settings.gradients ? 3 * np : 0;
        if (f->d_q32.bytes < sizeof(float) * (size_t)(nq + 1)) f->d_q32.alloc(sizeof(float) * (size_t)(nq + 1));
        if (f->d_out32.bytes < sizeof(float) * (size_t)(np + ng + 1))
            f->d_out32.alloc(sizeof(float) * (size_t)(np + ng + 1));
        cudaStream_t s = f->stream;
        if (nq) {
            CUDA_TRY(cudaMemcpyAsync(f->d_q32.ptr, charges, sizeof(float) * nq, cudaMemcpyHostToDevice, s));
            widen_kernel<<<grid_of(nq), 256, 0, s>>>(nq, f->d_q32.as<float>(), f->d_hq.as<double>());
            CUDA_TRY(cudaGetLastError());
        }
        const int rc = fmmgpu_helmholtz_evaluate_device(f, k_re, k_im, f->d_hq.as<double>(), f->d_hphi.as<double>(),
                                                        f->settings.gradients ? f->d_hg.as<double>() : nullptr);
        if (rc != FMMGPU_OK) throw Failure(rc, g_last_error);
        if (np) {
            float* o = f->d_out32.as<float>();
            narrow_kernel<<<grid_of(np), 256, 0, s>>>(np, f->d_hphi.as<double>(), o);
            if (ng) narrow_kernel<<<grid_of(ng), 256, 0, s>>>(ng, f->d_hg.as<double>(), o + np);
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaMemcpyAsync(potential, o, sizeof(float) * np, cudaMemcpyDeviceToHost, s));
            if (ng) CUDA_TRY(cudaMemcpyAsync(gradient, o + np, sizeof(float) * ng, cudaMemcpyDeviceToHost, s));
        }
        CUDA_TRY(cudaStreamSynchronize(s));
        if (f->eval->device_status()) throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
    });
}

double fmmgpu_helmholtz_table_seconds(const fmmgpu_fmm* f) { return f && f->eval ? f->eval->hh_table_seconds : 0.0; }

int fmmgpu_op_begin_evaluation(fmmgpu_fmm* f, const double* charges) {
    return guarded([&] {
        if (!f || !charges) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        if (f->mpass < f->settings.vectors)
            throw Failure(FMMGPU_UNSUPPORTED, "the level calls need every charge vector in one pass (device memory)");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const size_t m = f->settings.vectors, ns = f->plan.src_perm.size();
        CUDA_TRY(cudaMemcpyAsync(f->d_charges.ptr, charges, sizeof(double) * m * ns, cudaMemcpyHostToDevice, f->stream));
        f->eval->op_begin(f->d_charges.as<double>());
        f->op_begun = true;
    });
}

static int op_call(fmmgpu_fmm* f, int kind, int level) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        if (!f->op_begun) throw Failure(FMMGPU_INVALID_ARGUMENT, "no evaluation begun (fmmgpu_op_begin_evaluation)");
        if (level < 0 || level >= f->plan.nlevels)
            throw Failure(FMMGPU_INVALID_ARGUMENT, "level " + std::to_string(level) + " outside 0.." +
                                                       std::to_string(f->plan.nlevels - 1));
        CUDA_TRY(cudaSetDevice(f->settings.device));
        f->eval->op_level(kind, level);
    });
}

int fmmgpu_op_p2m(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_P2M, level); }
int fmmgpu_op_m2m(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_M2M, level); }
int fmmgpu_op_l2l(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_L2L, level); }
int fmmgpu_op_m2l(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_M2L, level); }
int fmmgpu_op_p2l(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_P2L, level); }
int fmmgpu_op_l2p(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_L2P, level); }
int fmmgpu_op_m2p(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_M2P, level); }
int fmmgpu_op_p2p(fmmgpu_fmm* f, int level) { return op_call(f, FMMGPU_OP_P2P, level); }

int fmmgpu_op_host_data(fmmgpu_fmm* f, int event) {
    (void)event;
    return guarded([&] {
        if (!f) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
    });
}

int fmmgpu_op_read_output(fmmgpu_fmm* f, double* potential, double* gradient) {
    return guarded([&] {
        if (!f || !potential || (f->settings.gradients && !gradient))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval || !f->op_begun) throw Failure(FMMGPU_INVALID_ARGUMENT, "no evaluation begun");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const size_t m = f->settings.vectors, nt = f->plan.tgt_perm.size();
        f->eval->op_output(f->d_phi.as<double>(), f->settings.gradients ? f->d_grad.as<double>() : nullptr);
        CUDA_TRY(cudaMemcpyAsync(potential, f->d_phi.ptr, sizeof(double) * m * nt, cudaMemcpyDeviceToHost, f->stream));
        if (f->settings.gradients)
            CUDA_TRY(cudaMemcpyAsync(gradient, f->d_grad.ptr, sizeof(double) * 3 * m * nt, cudaMemcpyDeviceToHost,
                                     f->stream));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        CUDA_TRY(cudaGetLastError());
        if (f->eval->device_status()) throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
    });
}

void* fmmgpu_fmm_stream(fmmgpu_fmm* f) { return f ? (void*)f->stream : nullptr; }

int fmmgpu_fmm_set_kind_timing(fmmgpu_fmm* f, int on) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        f->eval->timer.on = on != 0;
    });
}

int fmmgpu_fmm_set_m2l_path(fmmgpu_fmm* f, int path) {
    return guarded([&] {
        if (!f || !f->eval || path < 0 || path > 2) throw Failure(FMMGPU_INVALID_ARGUMENT, "invalid M2L path");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        f->eval->set_m2l_path(path);
        f->drop_graph();
    });
}

int fmmgpu_fmm_set_p2p_path(fmmgpu_fmm* f, int path) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        f->eval->set_p2p_path(path);
        f->drop_graph();
    });
}

int fmmgpu_helmholtz_m2l_tables(int p, double k, double half_width, double* tables) {
    return guarded([&] {
        if (!tables || p < 0 || p > 30 || !(k > 0.0) || !std::isfinite(k) || !(half_width > 0.0) ||
            !std::isfinite(half_width))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "need 0 <= p <= 30, a finite k > 0 and half-width > 0");
        std::vector<double> t;
        build_helmholtz_m2l_tables(p, k, half_width, t);
        std::copy(t.begin(), t.end(), tables);
    });
}

int fmmgpu_helmholtz_octant_tables(int p, double k, double half_width, double* m2m, double* l2l) {
    return guarded([&] {
        if (!m2m || !l2l || p < 0 || p > 30 || !(k > 0.0) || !std::isfinite(k) || !(half_width > 0.0) ||
            !std::isfinite(half_width))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "need 0 <= p <= 30, a finite k > 0 and half-width > 0");
        std::vector<double> a, b;
        build_helmholtz_octant_tables(p, k, half_width, a, b);
        std::copy(a.begin(), a.end(), m2m);
        std::copy(b.begin(), b.end(), l2l);
    });
}

int fmmgpu_fmm_set_kinds(fmmgpu_fmm* f, int kinds) {
    return guarded([&] {
        if (!f || !f->eval || kinds < 1 || kinds > 3) throw Failure(FMMGPU_INVALID_ARGUMENT, "invalid kinds");
        f->eval->kinds = kinds;
        f->drop_graph();
    });
}

int fmmgpu_fmm_set_overlap(fmmgpu_fmm* f, int on) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        f->eval->overlap = on != 0;
        f->drop_graph();
    });
}

int fmmgpu_fmm_set_graph(fmmgpu_fmm* f, int on) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        f->graph_on = on != 0;
        f->drop_graph();
    });
}

int fmmgpu_fmm_autotune(fmmgpu_fmm* f, const double* charges, int* choice) {
    return guarded([&] {
        if (!f || !charges) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (!f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "a plan-only handle cannot evaluate");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        const size_t m = f->settings.vectors, ns = f->plan.src_perm.size();
        CUDA_TRY(cudaMemcpyAsync(f->d_charges.ptr, charges, sizeof(double) * m * ns, cudaMemcpyHostToDevice, f->stream));
        f->drop_graph();
        f->eval->autotune(f->d_charges.as<double>(), f->d_phi.as<double>(),
                          f->settings.gradients ? f->d_grad.as<double>() : nullptr);
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        CUDA_TRY(cudaGetLastError());
        if (f->eval->device_status()) throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
        if (choice) {
            choice[0] = f->eval->p2p_warps;
            choice[1] = f->eval->leaf_block;
        }
    });
}

int fmmgpu_fmm_set_launch_shapes(fmmgpu_fmm* f, int p2p_warps, int leaf_block) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        if (p2p_warps != 1 && p2p_warps != 2 && p2p_warps != 4)
            throw Failure(FMMGPU_INVALID_ARGUMENT, "p2p_warps must be 1, 2 or 4");
        if (leaf_block != 32 && leaf_block != 64 && leaf_block != 128)
            throw Failure(FMMGPU_INVALID_ARGUMENT, "leaf_block must be 32, 64 or 128");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        f->eval->p2p_warps = p2p_warps;
        f->eval->leaf_block = leaf_block;
        f->drop_graph();
    });
}

int fmmgpu_fmm_set_vjp_store(fmmgpu_fmm* f, int on) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        if (on != 0 && on != 1) throw Failure(FMMGPU_INVALID_ARGUMENT, "on must be 0 or 1");
        if (on && !f->settings.gradients) throw Failure(FMMGPU_INVALID_ARGUMENT, "a VJP needs an FMM built with gradients");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        f->keep_valid = false;
        if (!on) {
            f->vjp_store = false;
            f->d_keep_q.alloc(0);
            f->d_keep_g.alloc(0);
            f->d_keep_flag.alloc(0);
            return;
        }
        const size_t m = f->settings.vectors, ns = f->plan.src_perm.size(), nt = f->plan.tgt_perm.size();
        const size_t bytes = sizeof(double) * m * (ns + 1) + sizeof(double) * 3 * m * (nt + 1);
        size_t free_b = 0, total_b = 0;
        CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        // memory asks for recomputation: the store may take at most half of what is free
        if (bytes > free_b / 2) throw Failure(FMMGPU_DEVICE_MEMORY, "no room to store the forward pass");
        f->d_keep_q.alloc(sizeof(double) * m * (ns + 1));
        f->d_keep_g.alloc(sizeof(double) * 3 * m * (nt + 1));
        f->d_keep_flag.alloc(sizeof(int));
        f->vjp_store = true;
    });
}

int fmmgpu_fmm_set_m2l_tile(fmmgpu_fmm* f, int tile) {
    return guarded([&] {
        if (!f || !f->eval) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        if (tile != 0 && tile != 1) throw Failure(FMMGPU_INVALID_ARGUMENT, "the M2L tile must be 0 or 1");
        if (tile == 1 && !f->eval->m2l_tile_columns(1))
            throw Failure(FMMGPU_INVALID_ARGUMENT, "this evaluator has no tensor-core M2L");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        f->eval->m2l_tile = tile;
        f->drop_graph();
    });
}

int fmmgpu_fmm_kind_times(fmmgpu_fmm* f, double* ms) {
    return guarded([&] {
        if (!f || !f->eval || !ms) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument or plan-only handle");
        CUDA_TRY(cudaSetDevice(f->settings.device));
        f->eval->timer.collect();
        for (int k = 0; k < kKinds; ++k) ms[k] = f->eval->timer.ms[k];
    });
}

int fmmgpu_fmm_synchronize(fmmgpu_fmm* f) {
    return guarded([&] {
        if (!f) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        CUDA_TRY(cudaStreamSynchronize(f->stream));
        CUDA_TRY(cudaGetLastError());
        if (f->eval && f->eval->device_status()) throw Failure(FMMGPU_DEVICE_ERROR, "a tensor-core wait timed out");
    });
}

int fmmgpu_fmm_info(const fmmgpu_fmm* f, fmmgpu_info* info) {
    return guarded([&] {
        if (!f || !info) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        const Plan& P = f->plan;
        info->nlevels = P.nlevels;
        info->nboxes = (int64_t)P.nboxes();
        info->nleaves = (int64_t)P.nleaves();
        info->nsources = (int64_t)P.src_perm.size();
        info->ntargets = (int64_t)P.tgt_perm.size();
        info->near_pairs = f->near_pairs;
        info->v_pairs = (int64_t)P.v.nnz();
        info->w_pairs = (int64_t)P.w.nnz();
        info->x_pairs = (int64_t)P.x.nnz();
        info->device_bytes = (int64_t)f->device_bytes;
        info->close_pairs = f->eval ? f->eval->close_pairs : 0;
        info->launches = f->eval ? f->eval->launches : 0;
        info->vectors_per_pass = f->eval ? f->mpass : 0;
        info->p2p_warps = f->eval ? f->eval->p2p_warps : 0;
        info->p2p_stream_bytes = f->eval ? f->eval->p2p_stream_bytes : 0;
        info->tables_loaded = f->tables_loaded;
        info->tuning_loaded = f->tuning_loaded;
        info->leaf_block = f->eval ? f->eval->leaf_block : 0;
        info->product_chunks = f->eval ? f->eval->product_chunks() : 0;
        info->m2l_tile_columns = f->eval ? f->eval->m2l_tile_columns(f->eval->m2l_tile) : 0;
        info->vjp_forward_reused = f->vjp_forward_reused;
    });
}

void fmmgpu_fmm_destroy(fmmgpu_fmm* f) {
    if (!f) return;
    if (f->eval || f->stream) cudaSetDevice(f->settings.device);
    if (f->stream) cudaStreamSynchronize(f->stream);
    if (f->transpose) fmmgpu_fmm_destroy(f->transpose);
    f->drop_graph();
    f->eval.reset();
    f->d_charges.alloc(0);
    f->d_phi.alloc(0);
    f->d_grad.alloc(0);
    if (f->h_status) cudaFreeHost(f->h_status);
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
}

int fmmgpu_fmm_boxes(const fmmgpu_fmm* f, uint64_t* keys, uint8_t* is_leaf) {
    return guarded([&] {
        if (!f) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        const Plan& P = f->plan;
        for (size_t b = 0; b < P.nboxes(); ++b) {
            if (keys) keys[b] = P.key[b];
            if (is_leaf) is_leaf[b] = P.box_leaf[b] >= 0;
        }
    });
}

int64_t fmmgpu_fmm_list(const fmmgpu_fmm* f, int kind, int64_t row, uint64_t* keys, int64_t cap) {
    if (!f) return -1;
    const Plan& P = f->plan;
    const Csr* c = kind == 0 ? &P.near : kind == 1 ? &P.v : kind == 2 ? &P.w : kind == 3 ? &P.x : nullptr;
    if (!c || row < 0 || row + 1 >= (int64_t)c->row.size()) return -1;
    int64_t n = c->row[row + 1] - c->row[row];
    for (int64_t e = 0; e < n && e < cap; ++e) {
        int32_t col = c->col[c->row[row] + e];
        int32_t box = (kind == 0 || kind == 3) ? P.leaf_box[col] : col;
        keys[e] = P.key[box];
    }
    return n;
}

int fmmgpu_fmm_tables(const fmmgpu_fmm* f, double* m2l, double* m2m, double* l2l) {
    return guarded([&] {
        if (!f) throw Failure(FMMGPU_INVALID_ARGUMENT, "null argument");
        if (m2l) std::memcpy(m2l, f->m2l.data(), f->m2l.size() * sizeof(double));
        if (m2m) std::memcpy(m2m, f->m2m.data(), f->m2m.size() * sizeof(double));
        if (l2l) std::memcpy(l2l, f->l2l.data(), f->l2l.size() * sizeof(double));
    });
}

const char* fmmgpu_status_string(int s) {
    switch (s) {
        case FMMGPU_OK: return "ok";
        case FMMGPU_INVALID_ARGUMENT: return "invalid argument";
        case FMMGPU_UNSUPPORTED: return "unsupported";
        case FMMGPU_DEVICE_MEMORY: return "device memory";
        case FMMGPU_DEVICE_ERROR: return "device error";
        case FMMGPU_NO_DEVICE: return "no device";
        default: return "unknown status";
    }
}

const char* fmmgpu_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
