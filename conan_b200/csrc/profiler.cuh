// profiler.cuh -- optional CUDA-event timing of every launch on a stream.
#pragma once

#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace conan {

// CONAN_DEBUG_SYNC=1: synchronise and check after every launch, no graphs.
inline bool debug_sync() {
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("CONAN_DEBUG_SYNC");
        v = (e && *e && *e != '0') ? 1 : 0;
    }
    return v == 1;
}

struct Profiler {
    bool on = false;
    std::vector<std::string> names;
    std::map<std::string, int> index;
    std::vector<double> total_ms;
    std::vector<int> launches;
    struct Rec {
        int k;
        cudaEvent_t a, b;
    };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;

    ~Profiler() {
        for (auto &r : pending) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    // Returns a record id (or -1 when off); call end() after the launch.
    int begin(const char *name, cudaStream_t s) {
        if (!on) return -1;
        auto it = index.find(name);
        int k;
        if (it == index.end()) {
            k = (int)names.size();
            index[name] = k;
            names.push_back(name);
            total_ms.push_back(0);
            launches.push_back(0);
        } else {
            k = it->second;
        }
        Rec r{k, take(), take()};
        cudaEventRecord(r.a, s);
        pending.push_back(r);
        return (int)pending.size() - 1;
    }
    void end(int rec, cudaStream_t s) {
        if (rec < 0) return;
        cudaEventRecord(pending[rec].b, s);
    }
    int collect() {
        for (auto &r : pending) {
            CONAN_CUDA(cudaEventSynchronize(r.b));
            float ms = 0;
            CONAN_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
            total_ms[r.k] += ms;
            launches[r.k] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
        return CONAN_OK;
    }
    void reset() {
        for (auto &t : total_ms) t = 0;
        for (auto &l : launches) l = 0;
    }
};

}  // namespace conan

// Launch `call` (a kernel launch or library call on stream S) bracketed by
// profiler events named NAME; checks the launch.
#define CONAN_TIMED(PROF, NAME, S, call)                                                   \
    do {                                                                                   \
        int rec_ = (PROF).begin((NAME), (S));                                              \
        call;                                                                              \
        CONAN_LAUNCHED();                                                                  \
        (PROF).end(rec_, (S));                                                             \
        if (::conan::debug_sync()) {                                                       \
            cudaError_t e_ = cudaStreamSynchronize(S);                                     \
            if (e_ != cudaSuccess)                                                         \
                return ::conan::set_error(CONAN_ERR_CUDA, "%s failed: %s (%s:%d)", (NAME),   \
                                          cudaGetErrorString(e_), __FILE__, __LINE__);     \
        }                                                                                  \
    } while (0)
