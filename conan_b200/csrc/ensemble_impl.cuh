// ensemble_impl.cuh -- batched ensembles of independent boxes with uneven
// mesh sizes (conan_ens_*). Included by pm.cu after the solver and the
// differentiable model.
//
// Members with the same mesh size and box form a class; a class is one
// batched solver (every kernel launch covers all its members, cuFFT runs
// batched), and each class runs on its own stream. conan_ens_run launches one
// CUDA graph that holds the whole n-step run of every class, the classes on
// parallel branches. The solver's autotuner picks the deposit and
// gradient-mesh kernels per class on the class's state half way through the
// run (clustered), then the initial state is restored.
#pragma once

#include <chrono>
#include <cstdio>
#include <string>

namespace conan {

// g = gscale (a - b), part[block] = sum (a - b)^2 (FP64, fixed order).
template <typename T>
__global__ void k_sqdiff(const T *__restrict__ a, const T *__restrict__ b, T *__restrict__ g, size_t n,
                         double gscale, double *__restrict__ part) {
    double s = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double d = (double)a[i] - (double)b[i];
        g[i] = (T)(gscale * d);
        s += d * d;
    }
    s = block_sum<double>(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

struct EnsBase {
    virtual ~EnsBase() {}
    virtual int init() = 0;
    virtual int run() = 0;
    virtual int forward_adjoint(double *loss) = 0;
    virtual int power_spectrum(int member, int nbins, double *k, double *P, double *cnt) = 0;
    virtual int state(int member, double *X, double *P) = 0;
    virtual int member_fields(int member, double *noise, double *target, double *gnoise) = 0;
    virtual int last_ms(double *run_ms, double *adj_ms) = 0;
    virtual size_t total_particles() const = 0;
    virtual std::string describe() const = 0;
    virtual int device() const = 0;
};

template <typename T, int R> struct Ens : EnsBase {
    struct Cls {
        int mbits = 0;
        double L = 0;
        std::vector<int> members;
        Diff<T, R> *d = nullptr;
        T *noise = nullptr, *tnoise = nullptr, *target = nullptr, *dens = nullptr, *gd = nullptr, *gn = nullptr;
        T *s0[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        cudaEvent_t join = nullptr, t0 = nullptr, t1 = nullptr;
        double tune_a = 0;  // scale factor of the state the autotuner timed (0: not tuned)
    };
    conan_ens_params prm{};
    std::vector<conan_ens_member> mem;
    std::vector<Cls> cls;
    std::vector<std::pair<int, int>> where;  // member -> (class, slot)
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr, e0 = nullptr, e1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    double run_ms = 0, adj_ms = 0;
    bool ready = false;
    bool have_grad = false;  // the noise gradients of a forward_adjoint are in gn

    ~Ens() override {
        if (main) cudaStreamSynchronize(main);
        if (graph) cudaGraphExecDestroy(graph);
        for (auto &c : cls) {
            if (c.join) cudaEventDestroy(c.join);
            if (c.t0) cudaEventDestroy(c.t0);
            if (c.t1) cudaEventDestroy(c.t1);
            delete c.d;
        }
        if (fork) cudaEventDestroy(fork);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (main) cudaStreamDestroy(main);
    }
    int device() const override { return prm.device; }

    int create(const conan_ens_params &p, int n, const conan_ens_member *m) {
        prm = p;
        mem.assign(m, m + n);
        where.resize(n);
        for (int i = 0; i < n; ++i) {
            int c = -1;
            for (size_t j = 0; j < cls.size(); ++j)
                if (cls[j].mbits == m[i].mbits && cls[j].L == m[i].size) c = (int)j;
            if (c < 0) {
                cls.emplace_back();
                c = (int)cls.size() - 1;
                cls[c].mbits = m[i].mbits;
                cls[c].L = m[i].size;
            }
            where[i] = {c, (int)cls[c].members.size()};
            cls[c].members.push_back(i);
        }
        CONAN_CUDA(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
        CONAN_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        CONAN_CUDA(cudaEventCreate(&e0));
        CONAN_CUDA(cudaEventCreate(&e1));
        for (auto &c : cls) {
            conan_diff_params dp{};
            dp.ic.dim = p.dim;
            dp.ic.mbits = c.mbits;
            dp.ic.size = c.L;
            dp.ic.scale_free = 1;
            dp.ic.smooth = 0;
            dp.ic.scale = p.scale;
            dp.ic.sigma = p.sigma;
            dp.ic.Omega0 = 0.32;
            dp.ic.H0 = 69.0;
            dp.ic.precision = p.precision;
            dp.ic.device = p.device;
            dp.pm.dim = p.dim;
            dp.pm.n_mass = 1 << c.mbits;
            dp.pm.f = 1;
            dp.pm.size = c.L;
            dp.pm.H0 = p.H0;
            dp.pm.Omega_m = p.Omega_m;
            dp.pm.Omega_L = p.Omega_L;
            dp.pm.precision = p.precision;
            dp.pm.gradient = CONAN_GRAD_FD4;
            dp.pm.device = p.device;
            dp.a0 = p.a0;
            dp.da = p.da;
            dp.n = p.n;
            dp.checkpoint_every = 8;
            std::vector<conan_ic_params> mic;
            for (int i : c.members) {
                conan_ic_params q = dp.ic;
                q.ns = mem[i].ns;
                q.seed = mem[i].seed;
                mic.push_back(q);
            }
            c.d = new Diff<T, R>();
            CONAN_TRY(c.d->create(dp, (int)c.members.size(), &mic));
            auto &pm = c.d->pm;
            CONAN_TRY(pm.alloc(&c.noise, pm.np));
            CONAN_TRY(pm.alloc(&c.tnoise, pm.np));
            CONAN_TRY(pm.alloc(&c.target, pm.mf.cells));
            CONAN_TRY(pm.alloc(&c.dens, pm.mf.cells));
            CONAN_TRY(pm.alloc(&c.gd, pm.mf.cells));
            CONAN_TRY(pm.alloc(&c.gn, pm.np));
            for (int k = 0; k < 2 * R; ++k) CONAN_TRY(pm.alloc(&c.s0[k], pm.np));
            CONAN_CUDA(cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming));
            CONAN_CUDA(cudaEventCreate(&c.t0));
            CONAN_CUDA(cudaEventCreate(&c.t1));
        }
        return CONAN_OK;
    }

    size_t total_particles() const override {
        size_t t = 0;
        for (auto &c : cls) t += c.d->pm.np;
        return t;
    }

    int save_state(Cls &c) {
        auto &pm = c.d->pm;
        for (int k = 0; k < R; ++k) {
            CONAN_CUDA(cudaMemcpyAsync(c.s0[k], pm.P.d[k], pm.np * sizeof(T), cudaMemcpyDeviceToDevice, pm.st));
            CONAN_CUDA(cudaMemcpyAsync(c.s0[R + k], pm.P.p[k], pm.np * sizeof(T), cudaMemcpyDeviceToDevice, pm.st));
        }
        return CONAN_OK;
    }
    int load_state(Cls &c) {
        auto &pm = c.d->pm;
        CONAN_TRY(pm.positions_reset());
        for (int k = 0; k < R; ++k) {
            CONAN_CUDA(cudaMemcpyAsync(pm.P.d[k], c.s0[k], pm.np * sizeof(T), cudaMemcpyDeviceToDevice, pm.st));
            CONAN_CUDA(cudaMemcpyAsync(pm.P.p[k], c.s0[R + k], pm.np * sizeof(T), cudaMemcpyDeviceToDevice, pm.st));
        }
        return CONAN_OK;
    }

    // Autotunes the class on a clustered state: the members are run half
    // way (n/2 steps from their initial state), the solver's autotuner times
    // its knobs there, and the initial state is put back.
    int tune(Cls &c) {
        auto &pm = c.d->pm;
        double a = prm.a0;
        CONAN_TRY(pm.steps(a, prm.da, 0, std::max(1u, prm.n / 2)));
        CONAN_TRY(pm.tune(a, prm.da));
        c.tune_a = a;
        return load_state(c);
    }

    int init() override {
        for (auto &c : cls) {
            auto &pm = c.d->pm;
            Mesh m1 = make_mesh(R, 1 << c.mbits, 1);
            for (size_t b = 0; b < c.members.size(); ++b) {
                const conan_ens_member &mb = mem[c.members[b]];
                CONAN_TRY(noise_device<T>(m1, mb.seed, c.noise + member_cells(m1, b), pm.st));
                CONAN_TRY(noise_device<T>(m1, mb.seed + 1000000ull, c.tnoise + member_cells(m1, b), pm.st));
            }
            CONAN_TRY(c.d->forward(c.tnoise, c.target, nullptr));  // target densities
            CONAN_TRY(c.d->initial_state(c.noise));
            CONAN_TRY(save_state(c));
            if (prm.autotune) CONAN_TRY(tune(c));
            CONAN_CUDA(cudaStreamSynchronize(pm.st));
            CONAN_TRY(pm.check_err());
        }
        ready = true;
        return CONAN_OK;
    }

    int build_graph() {
        for (auto &c : cls) {  // counts start at zero, as every replay leaves them
            auto &pm = c.d->pm;
            CONAN_CUDA(cudaStreamSynchronize(pm.st));
            CONAN_CUDA(cudaMemsetAsync(pm.count, 0, pm.mf.cells * sizeof(uint32_t), pm.st));
            CONAN_CUDA(cudaStreamSynchronize(pm.st));
            pm.ranks_pending = false;
        }
        cudaGraph_t g = nullptr;
        CONAN_CUDA(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
        int rc = CONAN_OK;
        cudaEventRecord(fork, main);
        for (auto &c : cls) {
            auto &pm = c.d->pm;
            cudaStreamWaitEvent(pm.st, fork, 0);
            if (rc == CONAN_OK) rc = load_state(c);
            double a = prm.a0;
            if (rc == CONAN_OK) rc = pm.steps(a, prm.da, 0, prm.n);
            cudaEventRecord(c.join, pm.st);
            cudaStreamWaitEvent(main, c.join, 0);
        }
        cudaError_t ce = cudaStreamEndCapture(main, &g);
        if (rc != CONAN_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return set_error(CONAN_ERR_CUDA, "ensemble graph capture failed: %s", cudaGetErrorString(ce));
        cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return set_error(CONAN_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ie));
        return CONAN_OK;
    }

    int run() override {
        if (!ready) return set_error(CONAN_ERR_STATE, "call conan_ens_init first");
        if (debug_sync()) {  // no graphs in the synchronous debug mode
            for (auto &c : cls) {
                CONAN_TRY(load_state(c));
                double a = prm.a0;
                CONAN_TRY(c.d->pm.steps(a, prm.da, 0, prm.n));
            }
            return CONAN_OK;
        }
        if (!graph) CONAN_TRY(build_graph());
        CONAN_CUDA(cudaEventRecord(e0, main));
        CONAN_CUDA(cudaGraphLaunch(graph, main));
        CONAN_CUDA(cudaEventRecord(e1, main));
        CONAN_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        CONAN_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        run_ms = ms;
        for (auto &c : cls) CONAN_TRY(c.d->pm.check_err());
        return CONAN_OK;
    }

    int forward_adjoint(double *loss) override {
        if (!ready) return set_error(CONAN_ERR_STATE, "call conan_ens_init first");
        double total = 0;
        for (auto &c : cls) {
            auto &pm = c.d->pm;
            CONAN_CUDA(cudaEventRecord(c.t0, pm.st));
            CONAN_TRY(c.d->forward(c.noise, c.dens, pm.st));
            const size_t nc1 = (size_t)1 << pm.mf.cshift;
            const int nb = 64;
            std::vector<double> h(nb);
            for (size_t b = 0; b < c.members.size(); ++b) {
                const size_t o = b * nc1;
                k_sqdiff<T><<<nb, 256, 0, pm.st>>>(c.dens + o, c.target + o, c.gd + o, nc1, 2.0 / (double)nc1,
                                                   c.d->part);
                CONAN_LAUNCHED();
                CONAN_CUDA(cudaMemcpyAsync(h.data(), c.d->part, nb * sizeof(double), cudaMemcpyDeviceToHost, pm.st));
                CONAN_CUDA(cudaStreamSynchronize(pm.st));
                double s = 0;
                for (int j = 0; j < nb; ++j) s += h[j];
                if (loss) loss[c.members[b]] = s / (double)nc1;
            }
            CONAN_TRY(c.d->backward(c.gd, c.gn, pm.st));
            CONAN_CUDA(cudaEventRecord(c.t1, pm.st));
        }
        for (auto &c : cls) {
            CONAN_CUDA(cudaEventSynchronize(c.t1));
            float ms = 0;
            CONAN_CUDA(cudaEventElapsedTime(&ms, c.t0, c.t1));
            total += ms;
            CONAN_TRY(c.d->pm.check_err());
        }
        adj_ms = total;
        have_grad = true;
        return CONAN_OK;
    }

    int power_spectrum(int member, int nbins, double *k, double *Pk, double *cnt) override {
        if (member < 0 || member >= (int)mem.size()) return set_error(CONAN_ERR_ARG, "no member %d", member);
        auto &c = cls[where[member].first];
        auto &pm = c.d->pm;
        CONAN_TRY(pm.deposit());
        CONAN_TRY(pm.fft.forward(pm.mesh, pm.spec));
        Mesh m1 = make_mesh(R, pm.mf.n, 1);
        CONAN_TRY(spectrum_bins<T>(pm.spec + (size_t)where[member].second * m1.mspec, m1, c.L, nbins, k, Pk, cnt,
                                   pm.st, nullptr));
        return pm.check_err();
    }

    int state(int member, double *X, double *Pm) override {
        if (member < 0 || member >= (int)mem.size()) return set_error(CONAN_ERR_ARG, "no member %d", member);
        auto &c = cls[where[member].first];
        auto &pm = c.d->pm;
        const size_t np1 = (size_t)1 << pm.P.bshift, o = (size_t)where[member].second * np1;
        Parts<T> v = pm.P;
        for (int k = 0; k < R; ++k) {
            v.d[k] += o;
            v.p[k] += o;
        }
        v.np = np1;
        return pm.export_state(v, np1, X, Pm);
    }

    int member_fields(int member, double *noise, double *target, double *gnoise) override {
        if (member < 0 || member >= (int)mem.size()) return set_error(CONAN_ERR_ARG, "no member %d", member);
        if (!ready) return set_error(CONAN_ERR_STATE, "call conan_ens_init first");
        if (gnoise && !have_grad) return set_error(CONAN_ERR_STATE, "no gradient: call conan_ens_forward_adjoint first");
        auto &c = cls[where[member].first];
        auto &pm = c.d->pm;
        const size_t n1 = (size_t)1 << pm.mf.cshift, o = (size_t)where[member].second * n1;
        std::vector<T> h(n1);
        const T *src[3] = {c.noise + o, c.target + o, c.gn + o};
        double *dst[3] = {noise, target, gnoise};
        CONAN_CUDA(cudaStreamSynchronize(pm.st));
        for (int f = 0; f < 3; ++f) {
            if (!dst[f]) continue;
            CONAN_CUDA(cudaMemcpy(h.data(), src[f], n1 * sizeof(T), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n1; ++i) dst[f][i] = (double)h[i];
        }
        return CONAN_OK;
    }

    int last_ms(double *r, double *a) override {
        if (r) *r = run_ms;
        if (a) *a = adj_ms;
        return CONAN_OK;
    }

    std::string describe() const override {
        std::string s = "{\"classes\": [";
        for (size_t i = 0; i < cls.size(); ++i) {
            const auto &c = cls[i];
            char buf[256];
            snprintf(buf, sizeof buf,
                     "%s{\"mesh\": %d, \"L\": %g, \"members\": %zu, \"deposit\": \"%s\", \"tuned_at_a\": %g, "
                     "\"tuning\": ",
                     i ? ", " : "", 1 << c.mbits, c.L, c.members.size(), c.d->pm.lag_on() ? "lagrangian" : "sorted",
                     c.tune_a);
            s += buf;
            s += c.d->pm.tune_report() + "}";
        }
        s += "]}";
        return s;
    }
};

inline EnsBase *make_ens(const conan_ens_params &p, int n, const conan_ens_member *m) {
    EnsBase *b = nullptr;
    int rc = CONAN_OK;
#define MAKE_ENS(T, R)              \
    {                               \
        auto *x = new Ens<T, R>();  \
        rc = x->create(p, n, m);    \
        b = x;                      \
    }
    if (p.precision == CONAN_FP32) {
        if (p.dim == 2) MAKE_ENS(float, 2) else MAKE_ENS(float, 3)
    } else {
        if (p.dim == 2) MAKE_ENS(double, 2) else MAKE_ENS(double, 3)
    }
#undef MAKE_ENS
    if (rc != CONAN_OK) {
        std::string msg = last_error();
        delete b;
        last_error() = msg;
        return nullptr;
    }
    return b;
}

}  // namespace conan
