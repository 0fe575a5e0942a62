// gnn_api.cu -- C ABI of the learned-preconditioner trainer: a set of training systems
// resident on one GPU, the network's parameters (FP32 master copy, Adam moments) and the
// forward / probe-loss / backward / Adam launches of gnn.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "common.hpp"
#include "gnn.hpp"

struct xplus_gnn_trainer {
    int device = 0;
    int probes = 1;
    cudaStream_t stream = nullptr;
    xplus::gnn::Arena arena;        // parameters, Adam moments, loss history
    xplus::gnn::Arena graph_arena;  // the resident training systems
    xplus::gnn::Arena work_arena;   // activations and temporaries, sized for the largest system
    std::vector<xplus::gnn::DevGraph> graphs;
    xplus::gnn::Work work;
    int work_n = 0, work_low = 0;
    int P = 0;
    int step = 0;
    float *master = nullptr, *wr = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    double* d_glow = nullptr;
    double* d_losses = nullptr;
    int losses_cap = 0;
    int max_glow = 0;
};

namespace xplus {
namespace {

void tcheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void trainer_destroy(xplus_gnn_trainer* t) {
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    t->graph_arena.release();
    t->work_arena.release();
    t->arena.release();
    if (t->stream) cudaStreamDestroy(t->stream);
    cudaGetLastError();
    delete t;
}

// Uploads the training systems, replacing any resident ones; the workspace grows to the largest
// system seen.  Parameters and the Adam state are kept.
void load_systems(xplus_gnn_trainer* t, int nsys, const int* const* row_ptrs, const int* const* col_idxs,
                  const double* const* values, const int* ns) {
    require(nsys > 0 && row_ptrs && col_idxs && values && ns, XPLUS_ERR_ARG, "null argument or nsys <= 0");
    tcheck(cudaStreamSynchronize(t->stream), "sync");
    t->graphs.clear();
    t->graph_arena.release();
    int max_n = 1, max_low = 1, max_glow = 1;
    for (int k = 0; k < nsys; ++k) {
        require(row_ptrs[k] && col_idxs[k] && values[k] && ns[k] > 0, XPLUS_ERR_ARG, "bad system " + std::to_string(k));
        validate_csr(ns[k], row_ptrs[k], col_idxs[k], row_ptrs[k][ns[k]]);
        gnn::HostGraph hg;
        hg.build(ns[k], row_ptrs[k], col_idxs[k], values[k]);
        gnn::DevGraph dg;
        dg.upload(hg, t->graph_arena, t->stream);
        tcheck(cudaStreamSynchronize(t->stream), "sync");  // host graph freed next
        t->graphs.push_back(dg);
        max_n = std::max(max_n, hg.n);
        max_low = std::max(max_low, hg.n_low);
        max_glow = std::max(max_glow, hg.n_glow);
    }
    if (max_n > t->work_n || max_low > t->work_low || max_glow > t->max_glow) {
        const int kind = t->work.loss_kind;
        t->work_arena.release();
        t->work_n = std::max(max_n, t->work_n);
        t->work_low = std::max(max_low, t->work_low);
        t->max_glow = std::max(max_glow, t->max_glow);
        t->work = gnn::Work();
        t->work.alloc(t->work_arena, t->work_n, t->work_low, t->probes, true);
        t->work.loss_kind = kind;
        t->d_glow = t->work_arena.get<double>(static_cast<size_t>(t->max_glow));
    }
}

// Steps [first, first + steps) of a cosine schedule from lr to lr_final over total steps; the
// resident systems in a seeded shuffle per epoch.
void train_window(xplus_gnn_trainer* t, int steps, double lr, double lr_final, uint64_t seed, int64_t first,
                  int64_t total, double* losses) {
    require(t && steps > 0 && lr > 0.0 && lr_final > 0.0, XPLUS_ERR_ARG, "bad argument");
    require(first >= 0 && total >= first + steps, XPLUS_ERR_ARG, "schedule window outside [0, total_steps)");
    tcheck(cudaSetDevice(t->device), "cudaSetDevice");
    cudaStream_t st = t->stream;
    if (steps > t->losses_cap) {
        t->d_losses = t->arena.get<double>(static_cast<size_t>(steps));
        t->losses_cap = steps;
    }
    const int ns = static_cast<int>(t->graphs.size());
    std::mt19937_64 rng(seed ^ (0x9E3779B97F4A7C15ull * static_cast<uint64_t>(first + 1)));
    std::vector<int> order(static_cast<size_t>(ns));
    for (int s = 0; s < steps; ++s) {
        if (s % ns == 0) {
            for (int k = 0; k < ns; ++k) order[static_cast<size_t>(k)] = k;
            std::shuffle(order.begin(), order.end(), rng);
        }
        const int sys = order[static_cast<size_t>(s % ns)];
        const int64_t sg = first + s;
        const double frac = total > 1 ? static_cast<double>(sg) / static_cast<double>(total - 1) : 1.0;
        const double lr_s = lr_final + 0.5 * (lr - lr_final) * (1.0 + std::cos(3.141592653589793 * frac));
        gnn::round_params(t->master, t->wr, t->P, st);
        gnn::forward(t->graphs[static_cast<size_t>(sys)], t->wr, t->work, true, st);
        gnn::loss_backward(t->graphs[static_cast<size_t>(sys)], t->wr, t->work, t->grad,
                           seed * 1000003ull + static_cast<uint64_t>(sg) + 1ull, st);
        tcheck(cudaMemcpyAsync(t->d_losses + s, t->work.loss, sizeof(double), cudaMemcpyDeviceToDevice, st), "D2D");
        gnn::adam_step(t->master, t->grad, t->m, t->v, t->P, static_cast<float>(lr_s), ++t->step, st);
    }
    if (losses)
        tcheck(cudaMemcpyAsync(losses, t->d_losses, static_cast<size_t>(steps) * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    tcheck(cudaStreamSynchronize(st), "sync");
}

void trainer_create(int nsys, const int* const* row_ptrs, const int* const* col_idxs, const double* const* values,
                    const int* ns, int probes, int device, xplus_gnn_trainer** out) {
    require(nsys > 0 && row_ptrs && col_idxs && values && ns && out, XPLUS_ERR_ARG, "null argument or nsys <= 0");
    require(probes >= 1 && probes <= 64, XPLUS_ERR_ARG, "probes must be in [1, 64]");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, "no CUDA device available (the trainer has no CPU path)");
    }
    require(device >= 0 && device < count, XPLUS_ERR_ARG, "device ordinal out of range");
    cudaDeviceProp prop;
    tcheck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    require(prop.major == 10, XPLUS_ERR_CUDA, "this build targets sm_100 (B200) devices only");
    tcheck(cudaSetDevice(device), "cudaSetDevice");
    auto* t = new xplus_gnn_trainer();
    t->device = device;
    t->probes = probes;
    try {
        tcheck(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        load_systems(t, nsys, row_ptrs, col_idxs, values, ns);
        t->P = gnn::param_offsets().total;
        const size_t P = static_cast<size_t>(t->P);
        t->master = t->arena.get<float>(P);
        t->wr = t->arena.get<float>(P);
        t->grad = t->arena.get<float>(P);
        t->m = t->arena.get<float>(P);
        t->v = t->arena.get<float>(P);
        tcheck(cudaMemsetAsync(t->master, 0, P * sizeof(float), t->stream), "memset");
        tcheck(cudaMemsetAsync(t->m, 0, P * sizeof(float), t->stream), "memset");
        tcheck(cudaMemsetAsync(t->v, 0, P * sizeof(float), t->stream), "memset");
        tcheck(cudaStreamSynchronize(t->stream), "sync");
        *out = t;
    } catch (...) {
        trainer_destroy(t);
        throw;
    }
}

void check_sys(xplus_gnn_trainer* t, int sys) {
    require(t, XPLUS_ERR_ARG, "null trainer");
    require(sys >= 0 && sys < static_cast<int>(t->graphs.size()), XPLUS_ERR_ARG, "system index out of range");
}

}  // namespace
}  // namespace xplus

using namespace xplus;

extern "C" {

int xplus_gnn_param_count(void) { return gnn::param_offsets().total; }

int xplus_gnn_trainer_create(int nsys, const int* const* row_ptrs, const int* const* col_idxs,
                             const double* const* values, const int* ns, int probes, int device,
                             xplus_gnn_trainer** out) {
    return guarded([&] { trainer_create(nsys, row_ptrs, col_idxs, values, ns, probes, device, out); });
}

int xplus_gnn_trainer_destroy(xplus_gnn_trainer* t) {
    return guarded([&] { trainer_destroy(t); });
}

int xplus_gnn_set_params(xplus_gnn_trainer* t, const float* params) {
    return guarded([&] {
        require(t && params, XPLUS_ERR_ARG, "null argument");
        tcheck(cudaSetDevice(t->device), "cudaSetDevice");
        const size_t bytes = static_cast<size_t>(t->P) * sizeof(float);
        tcheck(cudaMemcpyAsync(t->master, params, bytes, cudaMemcpyHostToDevice, t->stream), "H2D");
        tcheck(cudaMemsetAsync(t->m, 0, bytes, t->stream), "memset");
        tcheck(cudaMemsetAsync(t->v, 0, bytes, t->stream), "memset");
        tcheck(cudaStreamSynchronize(t->stream), "sync");
        t->step = 0;
    });
}

int xplus_gnn_get_params(xplus_gnn_trainer* t, float* params) {
    return guarded([&] {
        require(t && params, XPLUS_ERR_ARG, "null argument");
        tcheck(cudaSetDevice(t->device), "cudaSetDevice");
        tcheck(cudaMemcpyAsync(params, t->master, static_cast<size_t>(t->P) * sizeof(float), cudaMemcpyDeviceToHost, t->stream), "D2H");
        tcheck(cudaStreamSynchronize(t->stream), "sync");
    });
}

int xplus_gnn_loss_grad(xplus_gnn_trainer* t, int sys, uint64_t seed, double* loss, float* grad) {
    return guarded([&] {
        check_sys(t, sys);
        tcheck(cudaSetDevice(t->device), "cudaSetDevice");
        cudaStream_t st = t->stream;
        gnn::round_params(t->master, t->wr, t->P, st);
        gnn::forward(t->graphs[static_cast<size_t>(sys)], t->wr, t->work, true, st);
        gnn::loss_backward(t->graphs[static_cast<size_t>(sys)], t->wr, t->work, grad ? t->grad : nullptr, seed, st);
        if (loss) tcheck(cudaMemcpyAsync(loss, t->work.loss, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        if (grad) tcheck(cudaMemcpyAsync(grad, t->grad, static_cast<size_t>(t->P) * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
        tcheck(cudaStreamSynchronize(st), "sync");
    });
}

int xplus_gnn_set_loss(xplus_gnn_trainer* t, int kind) {
    return guarded([&] {
        require(t, XPLUS_ERR_ARG, "null trainer");
        require(kind == XPLUS_GNN_LOSS_PROBE || kind == XPLUS_GNN_LOSS_KAPORIN, XPLUS_ERR_ARG, "unknown loss kind");
        t->work.loss_kind = kind == XPLUS_GNN_LOSS_KAPORIN ? gnn::kLossKaporin : gnn::kLossProbe;
    });
}

int xplus_gnn_adam(xplus_gnn_trainer* t, const float* grad, double lr) {
    return guarded([&] {
        require(t && grad && lr > 0.0, XPLUS_ERR_ARG, "bad argument");
        tcheck(cudaSetDevice(t->device), "cudaSetDevice");
        cudaStream_t st = t->stream;
        tcheck(cudaMemcpyAsync(t->grad, grad, static_cast<size_t>(t->P) * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
        gnn::adam_step(t->master, t->grad, t->m, t->v, t->P, static_cast<float>(lr), ++t->step, st);
        tcheck(cudaStreamSynchronize(st), "sync");
    });
}

int xplus_gnn_train(xplus_gnn_trainer* t, int steps, double lr, double lr_final, uint64_t seed, double* losses) {
    return guarded([&] { train_window(t, steps, lr, lr_final, seed, 0, steps, losses); });
}

int xplus_gnn_train_window(xplus_gnn_trainer* t, int steps, double lr, double lr_final, uint64_t seed,
                           int64_t first_step, int64_t total_steps, double* losses) {
    return guarded([&] { train_window(t, steps, lr, lr_final, seed, first_step, total_steps, losses); });
}

int xplus_gnn_trainer_load(xplus_gnn_trainer* t, int nsys, const int* const* row_ptrs, const int* const* col_idxs,
                           const double* const* values, const int* ns) {
    return guarded([&] {
        require(t, XPLUS_ERR_ARG, "null trainer");
        tcheck(cudaSetDevice(t->device), "cudaSetDevice");
        load_systems(t, nsys, row_ptrs, col_idxs, values, ns);
    });
}

int xplus_gnn_predict(xplus_gnn_trainer* t, int sys, double* g_low, int64_t* n_glow) {
    return guarded([&] {
        check_sys(t, sys);
        const gnn::DevGraph& g = t->graphs[static_cast<size_t>(sys)];
        if (n_glow) *n_glow = g.n_glow;
        if (!g_low) return;
        tcheck(cudaSetDevice(t->device), "cudaSetDevice");
        cudaStream_t st = t->stream;
        gnn::round_params(t->master, t->wr, t->P, st);
        gnn::forward(g, t->wr, t->work, false, st);
        gnn::g_to_low(g, t->work, t->d_glow, st);
        tcheck(cudaMemcpyAsync(g_low, t->d_glow, static_cast<size_t>(g.n_glow) * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        tcheck(cudaStreamSynchronize(st), "sync");
    });
}

}  // extern "C"
