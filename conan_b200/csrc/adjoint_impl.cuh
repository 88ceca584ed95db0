// adjoint_impl.cuh -- the differentiable PM model (conan_diff_*): white noise
// -> initial conditions -> Zel'dovich start -> n leapfrog steps -> final CIC
// density, and its hand-written adjoint. Included by pm.cu after PM<T,R>.
//
// Forward step i (state s_i = (d_i, p_i) at the start of the step):
//   drift  d_{i+1} = d_i + cd_i p_i
//   kick   p_{i+1} = p_i - ck_i F(d_{i+1}),
//   F_j = sum_b W^g_b(x_j) G(c^g_b),  G = FD4(phi),  phi = Green * delta,
//   delta(c) = mass sum_j W^d(x_j, c) - 1
// (W^g: the gather's CIC weights with the reference's truncating origin,
// W^d: the deposit's weights). Adjoint of step i, given (dbar, pbar) of
// s_{i+1} and v = pbar:
//   dbar -= ck_i J^T v,   pbar = v + cd_i dbar,
//   (J^T v)_j = sum_b dW^g_b(x_j) (v_j . G(c^g_b))
//             + mass sum_b dW^d_b(x_j) rhobar(c^d_b),
//   rhobar = Green * ( -sum_k FD4_k(U_k) ),  U_k = gather-transpose deposit
//   of v_k (the Green operator is symmetric and FD4 antisymmetric).
// The state is run backwards reversibly (p_i = p_{i+1} + ck_i F(d_{i+1}),
// d_i = d_{i+1} - cd_i p_i) with the exact state restored from a checkpoint
// every k steps, which bounds the FP32 reversal error.
#pragma once

#include "ic.cuh"

namespace conan {

// dW_b/dx_k of the CIC weight of corner b, with a0 = 1 - a1 per axis.
template <typename T, int R> __device__ inline T dweight(const T *a0, const T *a1, int b, int k) {
    T z = ((b >> k) & 1) ? T(1) : T(-1);
#pragma unroll
    for (int l = 0; l < R; ++l)
        if (l != k) z *= ((b >> l) & 1) ? a1[l] : a0[l];
    return z;
}

// Deposit cell and weights of particle i exactly as the forward deposit
// forms them (the FP32 deposit position is rounded to 2^-21 cell).
template <typename T, int R>
__device__ inline void deposit_corner_frame(const Parts<T> &P, const Mesh &m, size_t i, const T *d, int *cell,
                                            T *a0, T *a1) {
    int q[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        if constexpr (sizeof(T) == 4) {
            uint32_t fr;
            Pay<float>::cell_frac(d[k], q[k], m.n - 1, &cell[k], &fr);
            a1[k] = (float)fr * 0x1p-21f;
        } else {
            double fr;
            Pay<double>::cell_frac(d[k], q[k], m.n - 1, &cell[k], &fr);
            a1[k] = fr;
        }
        a0[k] = T(1) - a1[k];
    }
}

template <int R> __device__ inline uint32_t corner_index(const int *o, int b, const Mesh &m) {
    uint32_t ci = 0;
#pragma unroll
    for (int k = R - 1; k >= 0; --k) ci = (ci << m.shift) | (uint32_t)((o[k] + ((b >> k) & 1)) & (m.n - 1));
    return ci;
}

// dbar_i = mass sum_b dW^d_b(x_i) deltabar(c_b): adjoint of the final deposit.
template <typename T, int R>
__global__ void k_adj_deposit_grad(Parts<T> P, Mesh m, const T *__restrict__ deltabar, double mass, T *db0, T *db1,
                                   T *db2) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    T d[3], a0[3], a1[3];
    int cell[3];
#pragma unroll
    for (int k = 0; k < R; ++k) d[k] = P.d[k][i];
    deposit_corner_frame<T, R>(P, m, i, d, cell, a0, a1);
    T g[3] = {T(0), T(0), T(0)};
    deltabar += cell_base(P, m, i);
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        T v = __ldg(deltabar + corner_index<R>(cell, b, m));
#pragma unroll
        for (int k = 0; k < R; ++k) g[k] += dweight<T, R>(a0, a1, b, k) * v;
    }
    T *db[3] = {db0, db1, db2};
#pragma unroll
    for (int k = 0; k < R; ++k) db[k][i] = (T)mass * g[k];
}

// Per-block maximum of |v| over all components.
template <typename T>
__global__ void k_absmax(const T *v0, const T *v1, const T *v2, size_t n, int R, double *part) {
    __shared__ double sm[32];
    double mx = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        mx = fmax(mx, fabs((double)v0[i]));
        if (R > 1) mx = fmax(mx, fabs((double)v1[i]));
        if (R > 2) mx = fmax(mx, fabs((double)v2[i]));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sm[w]);
        part[blockIdx.x] = r;
    }
}

// Fixed-point exponent S for the vector deposit: every cell sum of
// |v| w 2^S stays below 2^61 (gather weights with the truncating origin can
// reach 3 per axis).
__global__ void k_fix_exponent(const double *part, int nb, double np, int R, int *S) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mx = 0;
    for (int b = 0; b < nb; ++b) mx = fmax(mx, part[b]);
    if (!(mx > 0)) {
        *S = 0;
        return;
    }
    double lg = log2(mx) + log2(np) + 2.0 * R;
    int s = (int)floor(61.0 - lg);
    *S = max(-1000, min(1000, s));
}

// U_k(c) += v_k W^g_b for every particle and gather corner, in 64-bit
// fixed point (integer atomics: the sums are exact and order-independent).
template <typename T, int R>
__global__ void k_adj_vec_deposit(Parts<T> P, Mesh m, const T *v0, const T *v1, const T *v2, int periodic,
                                  const int *__restrict__ S, unsigned long long *U0, unsigned long long *U1,
                                  unsigned long long *U2) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    const T *vv[3] = {v0, v1, v2};
    unsigned long long *U[3] = {U0, U1, U2};
    int q[3], o[3];
    T a0[3], a1[3], v[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        gather_axis<T>(P.d[k][i], q[k], periodic != 0, &o[k], &a1[k]);
        a0[k] = T(1) - a1[k];
        v[k] = vv[k][i];
    }
    const int s = *S;
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        T z = 1;
#pragma unroll
        for (int k = 0; k < R; ++k) z *= ((b >> k) & 1) ? a1[k] : a0[k];
        size_t ci = cell_base(P, m, i) + corner_index<R>(o, b, m);
#pragma unroll
        for (int k = 0; k < R; ++k) {
            long long qv = __double2ll_rn(ldexp((double)v[k] * (double)z, s));
            if (qv) atomicAdd(U[k] + ci, (unsigned long long)qv);
        }
    }
}

// out(c) = -sum_k FD4_k(U_k)(c): the adjoint of the FD4 gradient, from the
// fixed-point meshes (scale 2^-S) or from real meshes (S == nullptr).
template <typename T, int R, typename UT>
__global__ void k_neg_div(const UT *U0, const UT *U1, const UT *U2, const int *S, T *out, Mesh m) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.cells) return;
    const UT *U[3] = {U0, U1, U2};
    const uint32_t mask = m.n - 1;
    const double sc = S ? ldexp(1.0, -*S) : 1.0;
    double acc = 0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int sh = k * m.shift;
        uint32_t ck = (c >> sh) & mask, rest = c & ~(mask << sh);
        auto at = [&](int o) -> double {
            UT x = U[k][rest | (((ck + o) & mask) << sh)];
            if constexpr (sizeof(UT) == 8 && !std::is_floating_point<UT>::value)
                return (double)(long long)x;
            else
                return (double)x;
        };
        acc += (at(-2) - at(2)) / 12.0 + (at(1) - at(-1)) * (2.0 / 3.0);
    }
    out[c] = (T)(-acc * sc);
}

// One adjoint step (see the file comment): updates dbar, pbar and runs the
// state back from s_{i+1} to s_i, using G = FD4 gradient at d_{i+1} and
// rhobar = Green * div.
template <typename T, int R>
__global__ void k_adj_step(Parts<T> P, Mesh m, const G4<T> *__restrict__ G, const T *__restrict__ rhobar,
                           T *pb0, T *pb1, T *pb2, T *db0, T *db1, T *db2, double ck, double cd, double mass,
                           int periodic) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    T *pbv[3] = {pb0, pb1, pb2}, *dbv[3] = {db0, db1, db2};
    T d[3], p[3], v[3], dbar[3];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        d[k] = P.d[k][i];
        p[k] = P.p[k][i];
        v[k] = pbv[k][i];
        dbar[k] = dbv[k][i];
    }
    int q[3], o[3], cell[3];
    T a0[3], a1[3], b0[3], b1[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        gather_axis<T>(d[k], q[k], periodic != 0, &o[k], &a1[k]);
        a0[k] = T(1) - a1[k];
    }
    T F[3] = {T(0), T(0), T(0)}, t1[3] = {T(0), T(0), T(0)}, t2[3] = {T(0), T(0), T(0)};
    const size_t cb = cell_base(P, m, i);
    G += cb;
    rhobar += cb;
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        G4<T> g = load_g4(G + corner_index<R>(o, b, m));
        T gv[3] = {g.x, g.y, g.z};
        T z = 1, vg = 0;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            z *= ((b >> k) & 1) ? a1[k] : a0[k];
            vg += v[k] * gv[k];
        }
#pragma unroll
        for (int k = 0; k < R; ++k) {
            F[k] += gv[k] * z;
            t1[k] += dweight<T, R>(a0, a1, b, k) * vg;
        }
    }
    deposit_corner_frame<T, R>(P, m, i, d, cell, b0, b1);
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        T r = __ldg(rhobar + corner_index<R>(cell, b, m));
#pragma unroll
        for (int k = 0; k < R; ++k) t2[k] += dweight<T, R>(b0, b1, b, k) * r;
    }
    const T tck = (T)ck, tcd = (T)cd, tm = (T)mass;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        T dbn = dbar[k] - tck * (t1[k] + tm * t2[k]);
        dbv[k][i] = dbn;
        pbv[k][i] = v[k] + tcd * dbn;
        T pold = p[k] + tck * F[k];
        P.p[k][i] = pold;
        P.d[k][i] = d[k] - tcd * pold;
    }
}

// ubar_k = cdz dbar_k + cpz pbar_k in place in dbar (particle i = mass cell i).
template <typename T>
__global__ void k_za_adjoint(T *db, const T *pb, size_t n, double cdz, double cpz) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) db[i] = (T)(cdz * (double)db[i] + cpz * (double)pb[i]);
}

struct DiffBase {
    virtual ~DiffBase() {}
    virtual int forward(const void *noise, void *density, void *stream) = 0;
    virtual int backward(const void *gdens, void *gnoise, void *stream) = 0;
    virtual int device() const = 0;
};

template <typename T, int R> struct Diff : DiffBase {
    typedef typename Cplx<T>::type CT;
    conan_diff_params prm{};
    PM<T, R> pm;
    Mesh mm{}, mm1{};  // mass meshes of the batch and of one member
    std::vector<conan_ic_params> ic;
    // initial conditions on the mass mesh
    T *w = nullptr, *ict = nullptr, *ict2 = nullptr;
    CT *ics = nullptr, *ics2 = nullptr;
    void *icwork = nullptr;
    FFTPair icfft;
    double *part = nullptr;
    // adjoint state
    T *db[3] = {nullptr, nullptr, nullptr}, *pb[3] = {nullptr, nullptr, nullptr};
    unsigned long long *U[3] = {nullptr, nullptr, nullptr};
    T *rhobar = nullptr;
    int *S = nullptr;
    std::vector<T *> ckpt;  // per checkpoint: d[0..R), p[0..R)
    std::vector<double> a_start;
    cudaEvent_t ev = nullptr;
    bool have_forward = false;

    ~Diff() override {
        if (pm.st) cudaStreamSynchronize(pm.st);
        icfft.destroy();
        if (ev) cudaEventDestroy(ev);
    }

    // `batch` equal boxes; member b's initial conditions use member_ic[b]
    // (default: p.ic for every member).
    int create(const conan_diff_params &p, int batch = 1,
               const std::vector<conan_ic_params> *member_ic = nullptr) {
        prm = p;
        CONAN_TRY(pm.create(p.pm, batch));
        mm = make_mesh(R, p.pm.n_mass, batch);
        mm1 = make_mesh(R, p.pm.n_mass, 1);
        ic.assign(batch, p.ic);
        if (member_ic) ic = *member_ic;
        CONAN_TRY(pm.alloc(&w, mm.cells));
        CONAN_TRY(pm.alloc(&ict, mm.cells));
        CONAN_TRY(pm.alloc(&ict2, mm.cells));
        CONAN_TRY(pm.alloc(&ics, mm.spec));
        CONAN_TRY(pm.alloc(&ics2, mm.spec));
        CONAN_TRY(pm.alloc(&part, 1024));
        CONAN_TRY(icfft.create(mm1, sizeof(T) == 8, 1));
        CONAN_TRY(pm.alloc((char **)&icwork, icfft.work_bytes ? icfft.work_bytes : 16));
        CONAN_TRY(icfft.bind(icwork, pm.st));
        for (int k = 0; k < R; ++k) {
            CONAN_TRY(pm.alloc(&db[k], pm.np));
            CONAN_TRY(pm.alloc(&pb[k], pm.np));
            CONAN_TRY(pm.alloc(&U[k], pm.mf.cells));
        }
        CONAN_TRY(pm.alloc(&rhobar, pm.mf.cells));
        CONAN_TRY(pm.alloc(&S, 1));
        unsigned k = p.checkpoint_every ? p.checkpoint_every : 1;
        for (unsigned i = 0; i <= p.n; i += k)
            for (int c = 0; c < 2 * R; ++c) {
                T *b = nullptr;
                CONAN_TRY(pm.alloc(&b, pm.np));
                ckpt.push_back(b);
            }
        a_start.resize(p.n + 1);
        double a = p.a0;
        for (unsigned i = 0; i <= p.n; ++i) {
            a_start[i] = a;
            a += p.da;  // LeapFrog::run accumulates a += da
        }
        CONAN_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        return CONAN_OK;
    }
    int device() const override { return prm.pm.device; }
    unsigned kev() const { return prm.checkpoint_every ? prm.checkpoint_every : 1; }
    dim3 gp() const { return dim3((unsigned)((pm.np + 255) / 256)); }

    int enter(void *stream) {
        if (stream) {
            CONAN_CUDA(cudaEventRecord(ev, (cudaStream_t)stream));
            CONAN_CUDA(cudaStreamWaitEvent(pm.st, ev, 0));
        }
        return CONAN_OK;
    }
    int leave(void *stream) {
        if (stream) {
            CONAN_CUDA(cudaEventRecord(ev, pm.st));
            CONAN_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, ev, 0));
            return CONAN_OK;
        }
        CONAN_CUDA(cudaStreamSynchronize(pm.st));
        return pm.check_err();
    }
    int save_ckpt(unsigned slot) {
        for (int k = 0; k < R; ++k) {
            CONAN_CUDA(cudaMemcpyAsync(ckpt[slot * 2 * R + k], pm.P.d[k], pm.np * sizeof(T), cudaMemcpyDeviceToDevice,
                                       pm.st));
            CONAN_CUDA(cudaMemcpyAsync(ckpt[slot * 2 * R + R + k], pm.P.p[k], pm.np * sizeof(T),
                                       cudaMemcpyDeviceToDevice, pm.st));
        }
        return CONAN_OK;
    }
    int load_ckpt(unsigned slot) {
        CONAN_TRY(pm.positions_reset());
        for (int k = 0; k < R; ++k) {
            CONAN_CUDA(cudaMemcpyAsync(pm.P.d[k], ckpt[slot * 2 * R + k], pm.np * sizeof(T), cudaMemcpyDeviceToDevice,
                                       pm.st));
            CONAN_CUDA(cudaMemcpyAsync(pm.P.p[k], ckpt[slot * 2 * R + R + k], pm.np * sizeof(T),
                                       cudaMemcpyDeviceToDevice, pm.st));
        }
        return CONAN_OK;
    }
    double cdz() const { return -prm.a0 / (pm.res_m * pm.res_f); }
    double cpz() const { return -(prm.a0 + prm.da / 2) / (pm.res_m * pm.res_f); }

    // Initial conditions of every member from the noise (device, batch) and
    // the Zel'dovich start of the particle state at (a0, a0 + da/2).
    int initial_state(const void *noise) {
        cudaStream_t st = pm.st;
        CONAN_CUDA(cudaMemcpyAsync(w, noise, mm.cells * sizeof(T), cudaMemcpyDeviceToDevice, st));
        CONAN_CUDA(cudaMemcpyAsync(ict, w, mm.cells * sizeof(T), cudaMemcpyDeviceToDevice, st));
        for (int b = 0; b < mm.batch; ++b) {  // initial conditions, member by member
            T *x = ict + member_cells(mm, b);
            CONAN_TRY(grf_device<T>(ic[b], mm1, x, ics, icfft, part, st));
            CONAN_TRY(potential_device<T>(mm1, ic[b].size, x, ics, icfft, st));
        }
        k_zeldovich<T, R><<<gp(), 256, 0, st>>>(pm.P, ict, mm, cdz(), cpz());
        CONAN_LAUNCHED();
        CONAN_TRY(pm.positions_reset());
        pm.a_pos = prm.a0;
        pm.a_mom = prm.a0 + prm.da / 2;
        return CONAN_OK;
    }

    int forward(const void *noise, void *density, void *stream) override {
        CONAN_TRY(enter(stream));
        cudaStream_t st = pm.st;
        CONAN_TRY(initial_state(noise));
        for (unsigned i = 0; i < prm.n; ++i) {
            if (i % kev() == 0) CONAN_TRY(save_ckpt(i / kev()));
            double a = a_start[i], am = a + prm.da / 2;
            CONAN_TRY(pm.gkd(false, 0, true, pm.coef_drift(a, prm.da), true));
            CONAN_TRY(pm.deposit_poisson(am));
            CONAN_TRY(pm.gkd(true, pm.coef_kick(am, prm.da), false, 0, false));
        }
        CONAN_TRY(pm.deposit());  // final density
        CONAN_CUDA(cudaMemcpyAsync(density, pm.mesh, pm.mf.cells * sizeof(T), cudaMemcpyDeviceToDevice, st));
        have_forward = true;
        return leave(stream);
    }

    // rhobar = Green(a) * (-sum_k FD4_k(U_k)) without touching the gradient mesh
    int adjoint_poisson(double am) {
        cudaStream_t st = pm.st;
        const Mesh &mf = pm.mf;
        unsigned gc = (unsigned)((mf.cells + 255) / 256);
        k_neg_div<T, R, unsigned long long><<<gc, 256, 0, st>>>(U[0], U[1], U[2], S, rhobar, mf);
        CONAN_LAUNCHED();
        // per-member normalisation: 1 / (cells of one box)
        double gsc = -pm.G / (am * (double)((size_t)1 << mf.cshift)) * std::pow(prm.pm.size / (2 * M_PI), 2);
        CONAN_TRY(pm.fft.forward(rhobar, pm.spec));
        CONAN_TRY(pm.green(pm.spec, gsc));
        CONAN_TRY(pm.fft.inverse(pm.spec, rhobar));
        return CONAN_OK;
    }

    int backward(const void *gdens, void *gnoise, void *stream) override {
        if (!have_forward) return set_error(CONAN_ERR_STATE, "backward without a forward call");
        CONAN_TRY(enter(stream));
        cudaStream_t st = pm.st;
        const Mesh &mf = pm.mf;
        const unsigned gc = (unsigned)((mf.cells + 255) / 256);
        // the density adjoint through the final deposit
        CONAN_CUDA(cudaMemcpyAsync(rhobar, gdens, mf.cells * sizeof(T), cudaMemcpyDeviceToDevice, st));
        k_adj_deposit_grad<T, R><<<gp(), 256, 0, st>>>(pm.P, mf, rhobar, pm.mass, db[0], db[1], db[2]);
        CONAN_LAUNCHED();
        for (int k = 0; k < R; ++k) CONAN_CUDA(cudaMemsetAsync(pb[k], 0, pm.np * sizeof(T), st));
        for (int i = (int)prm.n - 1; i >= 0; --i) {
            double a = a_start[i], am = a + prm.da / 2;
            double ck = pm.coef_kick(am, prm.da), cd = pm.coef_drift(a, prm.da);
            // forward force at d_{i+1}: deposit, potential, gradient mesh
            CONAN_TRY(pm.deposit_poisson(am));
            // U = gather-transpose deposit of v = pbar
            const int nb = 296;
            k_absmax<T><<<nb, 256, 0, st>>>(pb[0], pb[1], pb[2], pm.np, R, part);
            CONAN_LAUNCHED();
            k_fix_exponent<<<1, 32, 0, st>>>(part, nb, (double)pm.np, R, S);
            CONAN_LAUNCHED();
            for (int k = 0; k < R; ++k)
                CONAN_CUDA(cudaMemsetAsync(U[k], 0, mf.cells * sizeof(unsigned long long), st));
            k_adj_vec_deposit<T, R><<<gp(), 256, 0, st>>>(pm.P, mf, pb[0], pb[1], pb[2], prm.pm.periodic_gather, S,
                                                          U[0], U[1], U[2]);
            CONAN_LAUNCHED();
            CONAN_TRY(adjoint_poisson(am));
            k_adj_step<T, R><<<gp(), 256, 0, st>>>(pm.P, mf, pm.grad, rhobar, pb[0], pb[1], pb[2], db[0], db[1],
                                                   db[2], ck, cd, pm.mass, prm.pm.periodic_gather);
            CONAN_LAUNCHED();
            if ((unsigned)i % kev() == 0) CONAN_TRY(load_ckpt((unsigned)i / kev()));
        }
        // Zel'dovich, potential and random-field adjoints on the mass mesh
        unsigned gm = (unsigned)((mm.cells + 255) / 256);
        for (int k = 0; k < R; ++k) {
            k_za_adjoint<T><<<gm, 256, 0, st>>>(db[k], pb[k], mm.cells, cdz(), cpz());
            CONAN_LAUNCHED();
        }
        k_neg_div<T, R, T><<<gm, 256, 0, st>>>(db[0], db[1], db[2], nullptr, ict, mm);
        CONAN_LAUNCHED();
        for (int b = 0; b < mm.batch; ++b) {
            const size_t o = member_cells(mm, b);
            CONAN_TRY(potential_device<T>(mm1, ic[b].size, ict + o, ics, icfft, st));
            CONAN_TRY(grf_adjoint_device<T>(ic[b], mm1, w + o, ict + o, (T *)gnoise + o, ics, ics2, ict2, icfft,
                                            part, st));
        }
        (void)gc;
        return leave(stream);
    }
};

inline DiffBase *make_diff(const conan_diff_params &p) {
    DiffBase *b = nullptr;
    int rc = CONAN_OK;
#define MAKE_DIFF(T, R)               \
    {                                 \
        auto *x = new Diff<T, R>();   \
        rc = x->create(p);            \
        b = x;                        \
    }
    if (p.pm.precision == CONAN_FP32) {
        if (p.pm.dim == 1) MAKE_DIFF(float, 1) else if (p.pm.dim == 2) MAKE_DIFF(float, 2) else MAKE_DIFF(float, 3)
    } else {
        if (p.pm.dim == 1) MAKE_DIFF(double, 1) else if (p.pm.dim == 2) MAKE_DIFF(double, 2) else MAKE_DIFF(double, 3)
    }
#undef MAKE_DIFF
    if (rc != CONAN_OK) {
        std::string msg = last_error();
        delete b;
        last_error() = msg;
        return nullptr;
    }
    return b;
}

}  // namespace conan
