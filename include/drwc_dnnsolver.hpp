/* C++ mirror of the reference's dnnsolver classes over the C ABI of drwc.h.
 *
 * Replaces, at the source level, the classes of
 * inference_cpp/src/dnn_solver.h:43-201 (DNNSolver, DNNSolverPoisson,
 * DNNSolverGrad) and parallel_sampler.cpp:12-211 (ParallelSampler): the same
 * class and method names, the same std::vector<float> query layouts (15
 * layers x 2 floats and 15 cuboids x 7 floats per query, padding -9999) and
 * outputs (3 floats per Poisson query, 5 per first-hop query), the same
 * exceptions. Header-only; link with libdrwc.so. A caller built against the
 * reference header recompiles against this one (`using namespace
 * drwc_dnnsolver;`): it is not binary-compatible with the closed walker's
 * objects, whose class layouts hold libtorch members.
 *
 * Differences a caller sees:
 *   - the transition kernels are the FDM surface Green's function of the
 *     voxelised cube (drwc_transition_batch / drwc_first_hop_batch), so
 *     loadModels reads no model files;
 *   - draws come from Philox4x32-10 keyed by (seed, stream + query): the
 *     solver advances its stream by the batch size on every call, so a
 *     sequence of calls is reproducible;
 *   - structureConstruction returns host vectors (eps [n][N^3] normalised by
 *     each cube's maximum, and the maxima) instead of device tensors.
 */
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <future>
#include <iostream>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "drwc.h"

namespace drwc_dnnsolver {

constexpr int MAX_SAMPLES = 2048;  // dnn_solver.h:27-30
constexpr int MAX_CUBOIDS = 15;
constexpr int MAX_LAYERS = 15;
constexpr int PADDING_VALUE = -9999;
constexpr int kLayerStride = 2 * MAX_LAYERS;   // floats per query
constexpr int kCuboidStride = 7 * MAX_CUBOIDS;

enum class Axis : int { X = 0, Y = 1, Z = 2 };

inline void check_status(int rc, const char* what) {
    if (rc != DRWC_OK)
        throw std::runtime_error(std::string(what) + ": " + drwc_status_string(rc));
}

class DNNSolver {
   public:
    static constexpr int N = 23;
    static constexpr int NN = N * N;
    static constexpr int NNN = N * N * N;

    explicit DNNSolver(int device_idx = 0, uint64_t seed = 0x5EED) : seed_(seed) {
        check_status(drwc_ctx_create(device_idx, &ctx_), "drwc_ctx_create");
    }
    virtual ~DNNSolver() {
        if (ctx_) drwc_ctx_destroy(ctx_);
    }
    DNNSolver(const DNNSolver&) = delete;
    DNNSolver& operator=(const DNNSolver&) = delete;

    // Cubes of numSamples queries: eps [numSamples][N^3] (normalised by each
    // cube's maximum) and the maxima [numSamples].
    std::pair<std::vector<float>, std::vector<float>> structureConstruction(
        const std::vector<float>& layerStructures, const std::vector<float>& cuboidStructures,
        int numSamples, bool verbose = false) {
        queries(layerStructures, cuboidStructures, numSamples);
        std::pair<std::vector<float>, std::vector<float>> out;
        out.first.resize((size_t)numSamples * NNN);
        out.second.resize((size_t)numSamples);
        check_status(drwc_structure_construction(ctx_, numSamples, N, layerStructures.data(),
                                                 cuboidStructures.data(), 1, out.first.data(),
                                                 out.second.data()),
                     "drwc_structure_construction");
        if (verbose) std::cout << "structureConstruction: " << numSamples << " cubes\n";
        return out;
    }

    virtual void loadModels(bool verbose = false) = 0;
    virtual std::vector<float> sample(const std::vector<float>& layerStructures,
                                      const std::vector<float>& cuboidStructures) = 0;
    virtual std::vector<float> sample(const std::vector<float>& layerStructures,
                                      const std::vector<float>& cuboidStructures,
                                      const std::vector<int>& axis) = 0;

    drwc_ctx* context() const { return ctx_; }

   protected:
    // Query count of a batch; throws when the two arrays disagree.
    static int queries(const std::vector<float>& layers, const std::vector<float>& cuboids,
                       int expect = -1) {
        const size_t n = layers.size() / kLayerStride;
        if (layers.size() % kLayerStride || cuboids.size() != n * kCuboidStride ||
            (expect >= 0 && (size_t)expect != n))
            throw std::invalid_argument("layers must hold 30 and cuboids 105 floats per query");
        return (int)n;
    }
    uint64_t take_stream(int n) { return stream_.fetch_add((uint64_t)n); }

    drwc_ctx* ctx_ = nullptr;
    uint64_t seed_;
    std::atomic<uint64_t> stream_{0};
};

class DNNSolverPoisson : public DNNSolver {
   public:
    explicit DNNSolverPoisson(int device_idx = 0, uint64_t seed = 0x5EED)
        : DNNSolver(device_idx, seed) {}

    void loadModels(bool verbose = false) override {
        if (verbose) std::cout << "\tFDM transition kernels: no models to load\n";
    }

    // [x, y, z] in [-1, 1] per query (dnn_solver_poisson.cpp:35-63).
    std::vector<float> sample(const std::vector<float>& layerStructures,
                              const std::vector<float>& cuboidStructures) override {
        const int n = queries(layerStructures, cuboidStructures);
        std::vector<float> out((size_t)3 * n);
        if (n == 0) return out;
        check_status(drwc_transition_batch(ctx_, n, N, layerStructures.data(),
                                           cuboidStructures.data(), seed_, take_stream(n),
                                           out.data()),
                     "drwc_transition_batch");
        return out;
    }

    // The axis does not apply to the Green's function (dnn_solver_poisson.cpp:65-84).
    std::vector<float> sample(const std::vector<float>& layerStructures,
                              const std::vector<float>& cuboidStructures,
                              const std::vector<int>& axis) override {
        static std::atomic<bool> warned{false};
        if (!axis.empty() && !warned.exchange(true))
            std::cerr << "Warning: Axis parameter provided to Green's function solver but will "
                         "be ignored. (This warning will only be shown once)\n";
        return sample(layerStructures, cuboidStructures);
    }
};

class DNNSolverGrad : public DNNSolver {
   public:
    explicit DNNSolverGrad(int device_idx = 0, uint64_t seed = 0x5EED)
        : DNNSolver(device_idx, seed) {}

    void loadModels(bool verbose = false) override {
        if (verbose) std::cout << "\tFDM transition kernels: no models to load\n";
    }

    std::vector<float> sample(const std::vector<float>&, const std::vector<float>&) override {
        throw std::runtime_error("Gradient solver requires axis parameter");
    }

    // [x, y, z, weight, eps_centre] per query (dnn_solver_gradient.cpp:49-73, 111-163).
    std::vector<float> sample(const std::vector<float>& layerStructures,
                              const std::vector<float>& cuboidStructures,
                              const std::vector<int>& axis) override {
        const int n = queries(layerStructures, cuboidStructures);
        if (axis.size() != (size_t)n) throw std::invalid_argument("one axis per query");
        std::vector<float> out((size_t)5 * n);
        if (n == 0) return out;
        std::vector<int32_t> ax(axis.begin(), axis.end());
        check_status(drwc_first_hop_batch(ctx_, n, N, layerStructures.data(),
                                          cuboidStructures.data(), ax.data(), seed_,
                                          take_stream(n), out.data()),
                     "drwc_first_hop_batch");
        return out;
    }
};

// Cross-thread batching of single queries: submit() enqueues and returns a
// future; one worker thread takes up to batch_size queued queries (at most
// MAX_SAMPLES) per solver call and splits the result evenly. A solver
// exception, or a result that does not split evenly, reaches every future of
// its batch. Queries still queued at destruction are processed first.
class ParallelSampler {
   public:
    ParallelSampler(DNNSolver* solver, size_t sample_size, size_t batch_size)
        : solver_(solver), sample_size_(sample_size),
          batch_size_(batch_size < 1 ? 1 : (batch_size > MAX_SAMPLES ? MAX_SAMPLES : batch_size)) {
        if (!solver_) throw std::invalid_argument("Solver pointer cannot be null");
        worker_ = std::thread([this] { loop(); });
    }
    ~ParallelSampler() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            shutdown_ = true;
        }
        cv_.notify_all();
        if (worker_.joinable()) worker_.join();
    }
    ParallelSampler(const ParallelSampler&) = delete;
    ParallelSampler& operator=(const ParallelSampler&) = delete;

    std::future<std::vector<float>> submit(const std::vector<float>& layer,
                                           const std::vector<float>& cuboid) {
        return push(layer, cuboid, -1);
    }
    std::future<std::vector<float>> submit(const std::vector<float>& layer,
                                           const std::vector<float>& cuboid, const int axis) {
        return push(layer, cuboid, axis);
    }

   private:
    struct Task {
        std::vector<float> layer, cuboid;
        int axis;  // -1: none
        std::promise<std::vector<float>> promise;
    };

    std::future<std::vector<float>> push(const std::vector<float>& l, const std::vector<float>& c,
                                         int axis) {
        auto t = std::make_unique<Task>();
        t->layer = l;
        t->cuboid = c;
        t->axis = axis;
        auto f = t->promise.get_future();
        {
            std::lock_guard<std::mutex> lock(mu_);
            q_.push_back(std::move(t));
        }
        cv_.notify_one();
        return f;
    }

    void loop() {
        for (;;) {
            std::vector<std::unique_ptr<Task>> batch;
            {
                std::unique_lock<std::mutex> lock(mu_);
                cv_.wait(lock, [this] { return shutdown_ || !q_.empty(); });
                if (q_.empty()) return;  // shut down with nothing left
                while (!q_.empty() && batch.size() < batch_size_) {
                    batch.push_back(std::move(q_.front()));
                    q_.pop_front();
                }
            }
            process(batch);
        }
    }

    void process(std::vector<std::unique_ptr<Task>>& batch) {
        std::vector<float> a, b;
        std::vector<int> axes;
        bool has_axis = false;
        for (auto& t : batch) has_axis |= t->axis >= 0;
        for (auto& t : batch) {
            a.insert(a.end(), t->layer.begin(), t->layer.end());
            b.insert(b.end(), t->cuboid.begin(), t->cuboid.end());
            if (has_axis) axes.push_back(t->axis >= 0 ? t->axis : 0);
        }
        std::vector<float> res;
        try {
            res = has_axis ? solver_->sample(a, b, axes) : solver_->sample(a, b);
        } catch (...) {
            for (auto& t : batch) t->promise.set_exception(std::current_exception());
            return;
        }
        if (res.size() % batch.size()) {
            const auto e = std::make_exception_ptr(
                std::runtime_error("Result size doesn't match expected batch output size"));
            for (auto& t : batch) t->promise.set_exception(e);
            return;
        }
        const size_t w = res.size() / batch.size();
        for (size_t i = 0; i < batch.size(); ++i)
            batch[i]->promise.set_value(std::vector<float>(res.begin() + i * w,
                                                           res.begin() + (i + 1) * w));
    }

    DNNSolver* solver_;
    const size_t sample_size_;
    const size_t batch_size_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::unique_ptr<Task>> q_;
    bool shutdown_ = false;
    std::thread worker_;
};

}  // namespace drwc_dnnsolver
