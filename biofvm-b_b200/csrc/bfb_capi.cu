// bfb_capi.cu -- the C ABI (include/biofvm_b200.h): handles, coefficients,
// Dirichlet, bulk, agents, step sequencing and CUDA-graph replay.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bfb_aux.cuh"
#include "bfb_internal.cuh"
#include "bfb_sweeps.cuh"

namespace bfb {

static thread_local std::string g_last_error = "no error";

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    set_error(std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " + what);
    return e == cudaErrorMemoryAllocation ? BFB_ERR_OOM : BFB_ERR_CUDA;
}


// ---------------------------------------------------------------------------
// Thomas factors, host FP64, in the reference's operation order
// (BioFVM_parallel.cpp:780-912). The reference build fuses the axpy
// `denom[m] += c1*c[m-1]` (g++ -ffp-contract=fast); std::fma does the same.
// This file is compiled with -ffp-contract=off so nothing else is fused.
// ---------------------------------------------------------------------------
static void axis_factors(int n, int S, double dt, double dx, const double *D, const double *lam,
                         std::vector<double> &den, std::vector<double> &c, std::vector<double> &c1v) {
    den.assign((size_t)n * S, 0.0);
    c.assign((size_t)n * S, 0.0);
    c1v.assign(S, 0.0);
    for (int d = 0; d < S; ++d) {
        double c1 = D[d] * dt;
        c1 /= dx;
        c1 /= dx;
        double c2 = lam[d] * dt;
        c2 /= 3.0;
        double c3 = 1.0;
        c3 += c1;
        c3 += c1;
        c3 += c2;
        double c3a = 1.0;
        c3a += c1;
        c3a += c2;
        c1v[d] = c1;
        for (int m = 0; m < n; ++m) {
            c[(size_t)m * S + d] = -c1;
            den[(size_t)m * S + d] = c3;
        }
        den[d] = c3a;
        den[(size_t)(n - 1) * S + d] = c3a;
        if (n == 1) den[d] = 1.0 + c2;
        c[d] /= den[d];
        for (int m = 1; m < n; ++m) {
            den[(size_t)m * S + d] = std::fma(c1, c[(size_t)(m - 1) * S + d], den[(size_t)m * S + d]);
            c[(size_t)m * S + d] /= den[(size_t)m * S + d];
        }
    }
}

static int upload_table(bfb_env_s *env, void *dst, const std::vector<double> &v) {
    if (env->precision == BFB_FP64) {
        BFB_CUDA(cudaMemcpy(dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(v.size());
        for (size_t q = 0; q < v.size(); ++q) f[q] = (float)v[q];
        BFB_CUDA(cudaMemcpy(dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    return BFB_OK;
}

// A packed V*S host table (the reference layout) into a device array laid
// out like the field (rows at the pitch Lp), in the env's precision.
static int upload_pitched_table(bfb_env_s *env, void *dst, const std::vector<double> &v) {
    const size_t rows = (size_t)env->nx * env->ny, L = (size_t)env->nz * env->S;
    const size_t eb = env->elem;
    std::vector<float> f;
    const void *src = v.data();
    if (env->precision == BFB_FP32) {
        f.resize(v.size());
        for (size_t q = 0; q < v.size(); ++q) f[q] = (float)v[q];
        src = f.data();
    }
    BFB_CUDA(cudaMemcpy2D(dst, (size_t)env->Lp * eb, src, L * eb, L * eb, rows, cudaMemcpyHostToDevice));
    return BFB_OK;
}

// First row from which every table is bitwise constant up to row n-2, over
// all substrates (at least 1; n-1 when there is no such tail).
static int tail_start(const std::vector<std::vector<double>> &tabs, int n, int S) {
    int m0 = 1;
    for (const auto &t : tabs)
        for (int d = 0; d < S; ++d) {
            int m = n - 2;
            if (m < 1) return std::max(1, n - 1);
            while (m > 1 && t[(size_t)(m - 1) * S + d] == t[(size_t)(n - 2) * S + d]) --m;
            m0 = std::max(m0, m);
        }
    return m0;
}

// The device tables for one axis from the reference's factors (den, c).
//   FP64: den and c as they are, and RN(1/den) for the division (div_rcp).
//   FP32: 1/den as a hi+lo pair of floats, c1/den and c rounded once; the
//         deviation form of the FP32 kernels (bfb_sweeps.cuh) needs no c1.
static int upload_factors(bfb_env_s *env, int axis, int n, const std::vector<double> &den,
                          const std::vector<double> &c, const std::vector<double> &c1) {
    const int S = env->S;
    const size_t nS = (size_t)n * S;
    std::vector<std::vector<double>> tabs;
    if (env->precision == BFB_FP64) {
        std::vector<double> rcp(nS);
        for (size_t q = 0; q < nS; ++q) rcp[q] = 1.0 / den[q];
        tabs = {den, c, rcp};
    } else {
        std::vector<double> rh(nS), rl(nS), a(nS), cf(nS);
        for (int m = 0; m < n; ++m)
            for (int d = 0; d < S; ++d) {
                const size_t q = (size_t)m * S + d;
                const double r = 1.0 / den[q];
                rh[q] = (double)(float)r;
                rl[q] = (double)(float)(r - rh[q]);
                a[q] = (double)(float)(c1[d] / den[q]);
                cf[q] = (double)(float)c[q];
            }
        tabs = {rh, rl, a, cf};
    }
    const int m0 = tail_start(tabs, n, S);
    std::vector<double> flat, tail(4 * (size_t)S, 0.0);
    flat.reserve(4 * nS);
    for (size_t k = 0; k < 4; ++k) {
        if (k < tabs.size()) {
            flat.insert(flat.end(), tabs[k].begin(), tabs[k].end());
            if (m0 <= n - 2)
                for (int d = 0; d < S; ++d) tail[k * S + d] = tabs[k][(size_t)m0 * S + d];
        } else {
            flat.insert(flat.end(), nS, 0.0);
        }
    }
    // the head rows [0, m0) again, [table][substrate][row], rows padded to hpad
    const int hpad = (m0 + 3) / 4 * 4;
    std::vector<double> head(4 * (size_t)S * hpad, 0.0);
    for (size_t k = 0; k < tabs.size(); ++k)
        for (int d = 0; d < S; ++d)
            for (int m = 0; m < std::min(hpad, n); ++m) head[(k * S + d) * hpad + m] = tabs[k][(size_t)m * S + d];
    int st = upload_table(env, env->fac_tab[axis], flat);
    if (st) return st;
    st = upload_table(env, env->fac_tail[axis], tail);
    if (st) return st;
    st = upload_table(env, env->fac_head[axis], head);
    if (st) return st;
    env->fac_m0[axis] = m0;
    env->fac_hpad[axis] = hpad;
    return BFB_OK;
}

static int ensure_factors(bfb_env_s *env, double dt) {
    if (env->factors_valid && (env->freeze_factors || env->factor_dt == dt)) return BFB_OK;
    const int ns[3] = {env->nx_global ? env->nx_global : env->nx, env->ny, env->nz};  // a slab: the whole x line
    std::vector<double> den, c, c1;
    // the factor tables are only read by kernels on env->stream
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    for (int a = 0; a < 3; ++a) {
        axis_factors(ns[a], env->S, dt, env->dx, env->D.data(), env->lambda.data(), den, c, c1);
        int st = upload_factors(env, a, ns[a], den, c, c1);
        if (st) return st;
    }
    int st = upload_table(env, env->c1, c1);
    if (st) return st;
    // g = 1/(1 + c2), c2 = dt*lambda/3 (BioFVM_parallel.cpp:793-794), as hi, lo
    std::vector<double> g(2 * (size_t)env->S);
    for (int d = 0; d < env->S; ++d) {
        double c2 = env->lambda[d] * dt;
        c2 /= 3.0;
        const double gv = 1.0 / (1.0 + c2);
        g[d] = (double)(float)gv;
        g[env->S + d] = (double)(float)(gv - g[d]);
    }
    if ((st = upload_table(env, env->g, g))) return st;
    env->factors_valid = true;
    env->factor_dt = dt;
    env->epoch++;
    return BFB_OK;
}

template <typename T>
static SweepArgs<T> make_args(bfb_env_s *env, int axis, bool bulk, double dt) {
    SweepArgs<T> a;
    a.f = static_cast<T *>(env->field);
    a.fo = a.f;
    a.nx = env->nx;
    a.ny = env->ny;
    a.nz = env->nz;
    a.S = env->S;
    a.Lp = env->Lp;
    const int ns[3] = {env->nx_global ? env->nx_global : env->nx, env->ny, env->nz};
    const size_t nS = (size_t)ns[axis] * env->S;
    const T *tab = static_cast<const T *>(env->fac_tab[axis]);
    a.fac.t0 = tab;
    a.fac.t1 = tab + nS;
    a.fac.t2 = tab + 2 * nS;
    a.fac.t3 = tab + 3 * nS;
    a.fac.tail = static_cast<const T *>(env->fac_tail[axis]);
    a.fac.head = static_cast<const T *>(env->fac_head[axis]);
    a.fac.m0 = env->fac_m0[axis];
    a.fac.hpad = env->fac_hpad[axis];
    a.c1 = static_cast<const T *>(env->c1);
    a.g = static_cast<const T *>(env->g);
    for (int f = 0; f < 6; ++f) a.dir.face[f] = static_cast<const T *>(env->faces[f]);
    a.dir.mask = env->d_mask;
    a.dir.nx = env->nx;
    a.dir.ny = env->ny;
    a.dir.nz = env->nz;
    a.dir.S = env->S;
    a.dir.any = env->dir_any;
    a.bulk.A = static_cast<const T *>(env->bulkA);
    a.bulk.B = static_cast<const T *>(env->bulkB);
    a.bulk.dt = (T)dt;
    a.bulk.on = bulk && env->bulk_on;
    a.err = env->d_err;
    return a;
}

static const CUtensorMap *tma_map(bfb_env_s *env, int axis) {
    return (env->use_tma && env->tuning.tma[axis] && env->tma_ok[axis]) ? &env->tmap[axis] : nullptr;
}

// the field's x / y tensor maps for the current row-group counts
static void encode_field_maps(bfb_env_s *env) {
    for (int a = 0; a < 2; ++a) {
        const int chunks = env->tuning.chunks[a];
        env->tma_lines[a] = strided_tile_lines(a == 0 ? env->nx : env->ny, (int)env->elem, chunks);
        env->tma_ok[a] = make_sweep_tensor_map(&env->tmap[a], &env->tma_crow[a], env->field, (int)env->elem, a,
                                               env->nx, env->ny, env->nz, env->S, chunks, env->Lp,
                                               env->tma_lines[a]);
        const int n = a == 0 ? env->nx : env->ny;
        env->tmem_ok[a] = env->precision == BFB_FP64 && tmem_sweep_fits(n) &&
                          make_tmem_sweep_map(&env->tmem_map[a], env->field, a, env->nx, env->ny, env->Lp);
    }
}

// One LOD diffusion step; `bulk` fuses a preceding bulk source/sink update
// into the x-sweep load.
template <typename T>
static int launch_strided_env(bfb_env_s *env, int axis, bool bulk, double dt, cudaStream_t s) {
    const SweepArgs<T> a = make_args<T>(env, axis, bulk, dt);
    if constexpr (sizeof(T) == 8) {  // the tensor-memory tiles where the tuning asks for them
        if (env->use_tma && env->tuning.tma[axis] == 2 && env->tmem_ok[axis]) {
            const int st = launch_strided_tmem(a, strided_geometry(a, axis), &env->tmem_map[axis],
                                               &env->tmem_map[axis], axis == 0 && (a.dir.any || a.bulk.on), s);
            if (st != kNotApplicable) return st;
        }
    }
    return launch_strided<T>(a, axis, axis == 0, env->tuning.warps[axis], tma_map(env, axis), tma_map(env, axis),
                             env->tma_crow[axis], env->tma_lines[axis], s);
}

static int refuse_slab(const bfb_env_s *env) {
    return env->nx_global ? fail(BFB_ERR_UNSUPPORTED, "an x-slab env sweeps x through bfb_slab_x_forward and "
                                                      "bfb_slab_x_backward")
                          : BFB_OK;
}

template <typename T>
static int run_diffusion(bfb_env_s *env, double dt, bool bulk, cudaStream_t s) {
    if (int st = refuse_slab(env)) return st;
    int st = launch_strided_env<T>(env, 0, bulk, dt, s);
    if (st) return st;
    st = launch_strided_env<T>(env, 1, false, dt, s);
    if (st) return st;
    return launch_contig<T>(make_args<T>(env, 2, false, dt), env->tuning.warps[2],
                            env->use_tma != 0 && env->tuning.tma[2] != 0, s, env->tuning.chunks[2]);
}

template <typename T>
static int run_steps(bfb_env_s *env, double dt, int n, int flags, cudaStream_t s) {
    for (int q = 0; q < n; ++q) {
        int st = BFB_OK;
        if (flags & BFB_STEP_DIFFUSION) {
            st = run_diffusion<T>(env, dt, (flags & BFB_STEP_BULK) != 0, s);
        } else if (flags & BFB_STEP_BULK) {
            st = launch_bulk<T>(make_args<T>(env, 0, true, dt), env->Np, s);
        }
        if (st) return st;
        if (flags & BFB_STEP_CELLS) {
            st = launch_cells(env, s);
            if (st) return st;
        }
    }
    return BFB_OK;
}

static int run_steps_any(bfb_env_s *env, double dt, int n, int flags, cudaStream_t s) {
    return env->precision == BFB_FP64 ? run_steps<double>(env, dt, n, flags, s) : run_steps<float>(env, dt, n, flags, s);
}

// Hooks for the batched ensemble (bfb_batch.cu): the per-env state a step
// needs, and the per-axis kernel arguments and tile geometry.
int env_prepare_step(bfb_env_s *env, double dt, int flags) {
    BFB_CUDA(cudaSetDevice(env->device));
    if (int st = refuse_slab(env)) return st;
    if (flags & BFB_STEP_DIFFUSION) return ensure_factors(env, dt);
    return BFB_OK;
}

template <typename T>
SweepArgs<T> env_sweep_args(bfb_env_s *env, int axis, double dt) {
    return make_args<T>(env, axis, false, dt);
}
template SweepArgs<double> env_sweep_args<double>(bfb_env_s *, int, double);
template SweepArgs<float> env_sweep_args<float>(bfb_env_s *, int, double);

// One or more steps of the env on stream s, as bfb_simulate issues them (the
// batch's graph mode captures these per env).
int env_run_steps(bfb_env_s *env, double dt, int n, int flags, cudaStream_t s) {
    return run_steps_any(env, dt, n, flags, s);
}

int env_tile_plan(bfb_env_s *env, int elem, int Lp, StridedGeom *gx, StridedGeom *gy, ContigGeom *gz, int vb16[3]) {
    const bool base16 = (reinterpret_cast<uintptr_t>(env->field) & 15) == 0;
    gx->axis = 0;
    gx->n = env->nx;
    gx->P = (long long)env->ny * Lp;
    gx->slab_stride = 0;
    gx->n_slabs = 1;
    gx->ncb = (int)((gx->P + 31) / 32);
    gy->axis = 1;
    gy->n = env->ny;
    gy->P = Lp;
    gy->slab_stride = (long long)env->ny * Lp;
    gy->n_slabs = env->nx;
    gy->ncb = (int)((gy->P + 31) / 32);
    vb16[0] = base16 && (gx->P * elem) % 16 == 0;
    vb16[1] = base16 && (gy->P * elem) % 16 == 0 && (gy->slab_stride * elem) % 16 == 0;
    gz->nz = env->nz;
    gz->nrows = (long long)env->nx * env->ny;
    gz->Lp = Lp;
    if (!strided_smem(env->nx, elem, 1) || !strided_smem(env->ny, elem, 1) ||
        !contig_smem(env->nz, env->S, Lp, elem, 1, &gz->R, &gz->RS))
        return fail(BFB_ERR_UNSUPPORTED, "batch: an env's lines are too long for a shared-memory tile");
    vb16[2] = base16 && ((long long)Lp * elem) % 16 == 0 && ((long long)gz->RS * elem) % 16 == 0;
    return BFB_OK;
}

static void drop_graph(bfb_env_s *env) {
    if (env->graph_exec) cudaGraphExecDestroy(env->graph_exec);
    env->graph_exec = nullptr;
    env->graph_flags = -1;
}

static int check_env(bfb_env_s *env) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    BFB_CUDA(cudaSetDevice(env->device));
    return BFB_OK;
}

static int bulk_tabulate(bfb_env_s *env, const double *Sr, const double *T, const double *U) {
    // A = T*S and B = U + S as the reference rounds them
    // (BioFVM_microenvironment.cpp:1131-1142).
    const size_t N = env->N;
    std::vector<double> A(N), B(N);
    for (size_t e = 0; e < N; ++e) {
        A[e] = T[e] * Sr[e];
        B[e] = U[e] + Sr[e];
    }
    // laid out like the field (rows at its pitch), which the fused x load indexes
    // (row padding zero, so a whole-array pass leaves padded field entries finite)
    if (!env->bulkA) {
        BFB_CUDA(cudaMalloc(&env->bulkA, env->elem * env->Np));
        BFB_CUDA(cudaMemset(env->bulkA, 0, env->elem * env->Np));
    }
    if (!env->bulkB) {
        BFB_CUDA(cudaMalloc(&env->bulkB, env->elem * env->Np));
        BFB_CUDA(cudaMemset(env->bulkB, 0, env->elem * env->Np));
    }
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    int st = upload_pitched_table(env, env->bulkA, A);
    if (st) return st;
    return upload_pitched_table(env, env->bulkB, B);
}

}  // namespace bfb

using namespace bfb;

// The device error flag is sticky: once a kernel's bounded wait ran out, the
// env's field is not trustworthy and every later synchronize reports it.
int bfb::env_check_device_error(bfb_env_s *env) {
    int flag = 0;
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    BFB_CUDA(cudaMemcpy(&flag, env->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) return fail(BFB_ERR_WATCHDOG, "a device-side wait ran out of its iteration limit (data movement stalled)");
    return BFB_OK;
}


// ===========================================================================
extern "C" {

BFB_API const char *bfb_last_error(void) { return g_last_error.c_str(); }
BFB_API int bfb_version(void) { return 100; }

BFB_API int bfb_create(bfb_env *out, int nx, int ny, int nz, int n_substrates, double dx, int precision, int device) {
    if (!out) return fail(BFB_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (nx < 1 || ny < 1 || nz < 1 || n_substrates < 1)
        return fail(BFB_ERR_SIZE, "grid sizes and substrate count must be >= 1");
    if (!(dx > 0) || !std::isfinite(dx)) return fail(BFB_ERR_INVALID_ARG, "dx must be finite and > 0");
    if (precision != BFB_FP64 && precision != BFB_FP32) return fail(BFB_ERR_INVALID_ARG, "precision must be BFB_FP64 or BFB_FP32");
    const long long V = (long long)nx * ny * nz;
    if (V > 0x7fffffffLL) return fail(BFB_ERR_SIZE, "more than 2^31-1 voxels");
    int ndev = 0;
    BFB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(BFB_ERR_INVALID_ARG, "no such CUDA device");
    BFB_CUDA(cudaSetDevice(device));
    sweeps_prepare_device();

    bfb_env_s *env = new bfb_env_s();
    env->device = device;
    env->precision = precision;
    env->nx = nx;
    env->ny = ny;
    env->nz = nz;
    env->S = n_substrates;
    env->dx = dx;
    env->bbox[0] = env->bbox[1] = env->bbox[2] = 0.0;
    env->bbox[3] = nx * dx;
    env->bbox[4] = ny * dx;
    env->bbox[5] = nz * dx;
    env->elem = precision == BFB_FP64 ? 8 : 4;
    env->V = V;
    env->N = V * n_substrates;
    {   // rows padded to whole 16-byte vectors where nz*S elements are not (TMA needs 16-byte pitches)
        const long long L = (long long)nz * n_substrates, epv = 16 / (long long)env->elem;
        if (L > 0x7fffffffLL - epv) {
            delete env;
            return fail(BFB_ERR_SIZE, "nz * substrates too large");
        }
        env->Lp = (int)((L + epv - 1) / epv * epv);
        env->Np = (long long)nx * ny * env->Lp;
    }
    env->D.assign(n_substrates, 0.0);
    env->lambda.assign(n_substrates, 0.0);
    env->activation.assign(n_substrates, 0);
    env->face_mask.assign(6 * (size_t)n_substrates, 0);
    int st = BFB_OK;
    auto alloc = [&](void **p, size_t bytes) {
        if (st) return;
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 1);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMalloc");
    };
    alloc(&env->field, env->elem * env->Np);
    const int ns[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        alloc(&env->fac_tab[a], env->elem * 4 * (size_t)ns[a] * n_substrates);
        alloc(&env->fac_tail[a], env->elem * 4 * (size_t)n_substrates);
        alloc(&env->fac_head[a], env->elem * 4 * (size_t)n_substrates * ((ns[a] + 3) / 4 * 4));
    }
    alloc(&env->c1, env->elem * n_substrates);
    alloc(&env->g, env->elem * 2 * n_substrates);
    alloc((void **)&env->d_mask, n_substrates);
    alloc((void **)&env->d_err, sizeof(int));
    if (!st) {
        cudaError_t e = cudaMemset(env->d_err, 0, sizeof(int));
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemset");
    }
    if (!st) encode_field_maps(env);
    if (!st) {
        cudaError_t e = cudaStreamCreateWithFlags(&env->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaStreamCreateWithFlags");
        env->stream = env->own_stream;
    }
    if (!st) {
        cudaError_t e = cudaMemset(env->field, 0, env->elem * env->Np);
        if (e == cudaSuccess) e = cudaMemset(env->d_mask, 0, n_substrates);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemset");
    }
    if (st) {
        bfb_destroy(env);
        return st;
    }
    *out = env;
    return BFB_OK;
}

BFB_API int bfb_create_domain(bfb_env *out, double x0, double x1, double y0, double y1, double z0, double z1,
                              double dx, int n_substrates, int precision, int device) {
    if (!out) return fail(BFB_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!(dx > 0) || !std::isfinite(dx)) return fail(BFB_ERR_INVALID_ARG, "dx must be finite and > 0");
    // BioFVM_parallel.cpp:100-102; counts outside int range (or from non-finite
    // extents) are rejected before the conversion
    const double eps = 1e-16;
    const double cx = std::ceil(eps + (x1 - x0) / dx), cy = std::ceil(eps + (y1 - y0) / dx),
                 cz = std::ceil(eps + (z1 - z0) / dx);
    for (double c : {cx, cy, cz})
        if (!(c >= 1.0 && c <= 2147483647.0))
            return fail(BFB_ERR_SIZE, "domain extents must be finite with x1 >= x0, y1 >= y0, z1 >= z0 and give "
                                      "at most 2^31-1 voxels per axis");
    const int nx = (int)cx, ny = (int)cy, nz = (int)cz;
    int st = bfb_create(out, nx, ny, nz, n_substrates, dx, precision, device);
    if (st) return st;
    bfb_env_s *env = *out;
    env->bbox[0] = x0;
    env->bbox[1] = y0;
    env->bbox[2] = z0;
    env->bbox[3] = x1;
    env->bbox[4] = y1;
    env->bbox[5] = z1;
    return BFB_OK;
}

BFB_API int bfb_destroy(bfb_env env) {
    if (!env) return BFB_OK;
    cudaSetDevice(env->device);
    if (env->stream) cudaStreamSynchronize(env->stream);
    drop_graph(env);
    agents_free(env);
    cudaFree(env->field);
    cudaFree(env->staging);
    for (int a = 0; a < 3; ++a) {
        cudaFree(env->fac_tab[a]);
        cudaFree(env->fac_tail[a]);
        cudaFree(env->fac_head[a]);
    }
    cudaFree(env->c1);
    cudaFree(env->g);
    for (int f = 0; f < 6; ++f) cudaFree(env->faces[f]);
    cudaFree(env->d_mask);
    cudaFree(env->bulkA);
    cudaFree(env->bulkB);
    cudaFree(env->partials);
    cudaFree(env->d_err);
    cudaFree(env->adj_ws);
    if (env->own_stream) cudaStreamDestroy(env->own_stream);
    delete env;
    return BFB_OK;
}

BFB_API int bfb_get_shape(bfb_env env, int *nx, int *ny, int *nz, int *S) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    if (nx) *nx = env->nx;
    if (ny) *ny = env->ny;
    if (nz) *nz = env->nz;
    if (S) *S = env->S;
    return BFB_OK;
}

BFB_API int bfb_set_stream(bfb_env env, void *stream) {
    int st = check_env(env);
    if (st) return st;
    // NULL selects the env's own stream again
    cudaStream_t want = stream ? (cudaStream_t)stream : env->own_stream;
    if (env->stream != want) {
        BFB_CUDA(cudaStreamSynchronize(env->stream));
        drop_graph(env);
    }
    env->stream = want;
    return BFB_OK;
}

BFB_API int bfb_set_option(bfb_env env, int option, int value) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    switch (option) {
    case BFB_OPT_FREEZE_FACTORS: env->freeze_factors = value != 0; break;
    case BFB_OPT_USE_GRAPHS:
        env->use_graphs = value != 0;
        drop_graph(env);
        break;
    case BFB_OPT_USE_TMA:
        env->use_tma = value != 0;
        drop_graph(env);
        break;
    default: return fail(BFB_ERR_INVALID_ARG, "unknown option");
    }
    return BFB_OK;
}

BFB_API int bfb_synchronize(bfb_env env) {
    int st = check_env(env);
    if (st) return st;
    return env_check_device_error(env);
}

BFB_API int bfb_watchdog_selftest(bfb_env env, int polls) {
    int st = check_env(env);
    if (st) return st;
    if (polls < 1 || polls > (1 << 20)) return fail(BFB_ERR_INVALID_ARG, "polls must be in [1, 2^20]");
    return launch_watchdog_probe(polls, env->d_err, env->stream);
}

BFB_API int bfb_set_coefficients(bfb_env env, const double *D, const double *lambda) {
    int st = check_env(env);
    if (st) return st;
    if (!D || !lambda) return fail(BFB_ERR_INVALID_ARG, "D and lambda must not be NULL");
    env->D.assign(D, D + env->S);
    env->lambda.assign(lambda, lambda + env->S);
    env->factors_valid = false;
    return BFB_OK;
}

static int ensure_staging(bfb_env_s *env) {
    if (env->staging) return BFB_OK;
    BFB_CUDA(cudaMalloc(&env->staging, sizeof(double) * env->N));
    return BFB_OK;
}

// Field transfers between the packed V*S reference layout (host or device
// buffers) and the env's field, whose rows may be padded (bfb_env_s::Lp).
// Same element type: one copy (2-D when the rows are padded).
static int copy_rows(bfb_env_s *env, void *dst, bool dst_is_field, const void *src, cudaMemcpyKind kind,
                     size_t eb, cudaStream_t s) {
    const size_t rows = (size_t)env->nx * env->ny, w = (size_t)env->nz * env->S * eb, pitched = (size_t)env->Lp * eb;
    if (pitched == w) {
        BFB_CUDA(cudaMemcpyAsync(dst, src, rows * w, kind, s));
    } else {
        BFB_CUDA(cudaMemcpy2DAsync(dst, dst_is_field ? pitched : w, src, dst_is_field ? w : pitched, w, rows, kind, s));
    }
    return BFB_OK;
}
// Device conversion between FP64 and FP32, packed <-> field layout.
static int convert_rows(bfb_env_s *env, const void *src, int src_prec, void *dst, bool dst_is_field, cudaStream_t s) {
    const long long rows = (long long)env->nx * env->ny;
    const int L = env->nz * env->S;
    const int sp = dst_is_field ? L : env->Lp, dp = dst_is_field ? env->Lp : L;
    if (src_prec == BFB_FP64)
        return launch_convert_d2f_rows((const double *)src, (float *)dst, rows, L, sp, dp, s);
    return launch_convert_f2d_rows((const float *)src, (double *)dst, rows, L, sp, dp, s);
}
// host doubles (packed) -> the field, converting on the device for FP32
static int field_from_host_doubles(bfb_env_s *env, const double *host, cudaStream_t s) {
    if (env->precision == BFB_FP64) return copy_rows(env, env->field, true, host, cudaMemcpyHostToDevice, 8, s);
    int st = ensure_staging(env);
    if (st) return st;
    BFB_CUDA(cudaMemcpyAsync(env->staging, host, sizeof(double) * env->N, cudaMemcpyHostToDevice, s));
    return convert_rows(env, env->staging, BFB_FP64, env->field, true, s);
}
// the field -> host doubles (packed)
static int field_to_host_doubles(bfb_env_s *env, double *host, cudaStream_t s) {
    if (env->precision == BFB_FP64) return copy_rows(env, host, false, env->field, cudaMemcpyDeviceToHost, 8, s);
    int st = ensure_staging(env);
    if (st) return st;
    if ((st = convert_rows(env, env->field, BFB_FP32, env->staging, false, s))) return st;
    BFB_CUDA(cudaMemcpyAsync(host, env->staging, sizeof(double) * env->N, cudaMemcpyDeviceToHost, s));
    return BFB_OK;
}

BFB_API int bfb_set_field(bfb_env env, const double *host) {
    int st = check_env(env);
    if (st) return st;
    if (!host) return fail(BFB_ERR_INVALID_ARG, "host is NULL");
    if ((st = field_from_host_doubles(env, host, env->stream))) return st;
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    return BFB_OK;
}

BFB_API int bfb_get_field(bfb_env env, double *host) {
    int st = check_env(env);
    if (st) return st;
    if (!host) return fail(BFB_ERR_INVALID_ARG, "host is NULL");
    if ((st = field_to_host_doubles(env, host, env->stream))) return st;
    return env_check_device_error(env);
}

BFB_API int bfb_set_field_raw(bfb_env env, const void *host) {
    int st = check_env(env);
    if (st) return st;
    if (!host) return fail(BFB_ERR_INVALID_ARG, "host is NULL");
    if ((st = copy_rows(env, env->field, true, host, cudaMemcpyHostToDevice, env->elem, env->stream))) return st;
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    return BFB_OK;
}

BFB_API int bfb_get_field_raw(bfb_env env, void *host) {
    int st = check_env(env);
    if (st) return st;
    if (!host) return fail(BFB_ERR_INVALID_ARG, "host is NULL");
    if ((st = copy_rows(env, host, false, env->field, cudaMemcpyDeviceToHost, env->elem, env->stream))) return st;
    return env_check_device_error(env);
}

// Device-to-device field transfer with precision conversion.
BFB_API int bfb_set_field_device(bfb_env env, const void *src, int src_precision) {
    int st = check_env(env);
    if (st) return st;
    if (!src) return fail(BFB_ERR_INVALID_ARG, "src is NULL");
    if (src_precision != BFB_FP64 && src_precision != BFB_FP32) return fail(BFB_ERR_INVALID_ARG, "bad precision");
    if (src_precision == env->precision) {
        if ((st = copy_rows(env, env->field, true, src, cudaMemcpyDeviceToDevice, env->elem, env->stream))) return st;
    } else {
        if ((st = convert_rows(env, src, src_precision, env->field, true, env->stream))) return st;
    }
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    return BFB_OK;
}

BFB_API int bfb_get_field_device(bfb_env env, void *dst, int dst_precision) {
    int st = check_env(env);
    if (st) return st;
    if (!dst) return fail(BFB_ERR_INVALID_ARG, "dst is NULL");
    if (dst_precision != BFB_FP64 && dst_precision != BFB_FP32) return fail(BFB_ERR_INVALID_ARG, "bad precision");
    if (dst_precision == env->precision) {
        if ((st = copy_rows(env, dst, false, env->field, cudaMemcpyDeviceToDevice, env->elem, env->stream))) return st;
    } else {
        if ((st = convert_rows(env, env->field, env->precision, dst, false, env->stream))) return st;
    }
    return env_check_device_error(env);
}

BFB_API int bfb_compare_fields(bfb_env test, bfb_env ref, double *out4) {
    int st = check_env(test);
    if (st) return st;
    if (!ref || !out4) return fail(BFB_ERR_INVALID_ARG, "null argument");
    if (test->nx != ref->nx || test->ny != ref->ny || test->nz != ref->nz || test->S != ref->S ||
        test->device != ref->device)
        return fail(BFB_ERR_SIZE, "fields differ in shape or device");
    BFB_CUDA(cudaStreamSynchronize(ref->stream));
    return compare_fields(test->field, test->precision, test->Lp, ref->field, ref->precision, ref->Lp,
                          (long long)test->nx * test->ny, test->nz * test->S, out4, test->stream);
}

BFB_API int bfb_field_device_ptr(bfb_env env, void **dptr) {
    if (!env || !dptr) return fail(BFB_ERR_INVALID_ARG, "null argument");
    *dptr = env->field;
    return BFB_OK;
}

BFB_API int bfb_field_pitch(bfb_env env, int *row_elems) {
    if (!env || !row_elems) return fail(BFB_ERR_INVALID_ARG, "null argument");
    *row_elems = env->Lp;
    return BFB_OK;
}

// Dirichlet: cut the six face arrays out of per-voxel values.
static int dirichlet_install(bfb_env_s *env, const std::vector<double> *faces_host /* 6 arrays or null */,
                             const uint8_t *activation, const uint8_t *face_mask) {
    const int S = env->S;
    if (activation) env->activation.assign(activation, activation + S);
    for (int f = 0; f < 6; ++f)
        for (int d = 0; d < S; ++d) {
            const uint8_t base = face_mask ? face_mask[f * S + d] : 1;
            env->face_mask[f * S + d] = (base && env->activation[d]) ? 1 : 0;
            // a slab holds the grid's x faces only at its ends of the grid
            if (env->nx_global && ((f == 0 && env->x0 != 0) || (f == 1 && env->x0 + env->nx != env->nx_global)))
                env->face_mask[f * S + d] = 0;
        }
    std::vector<uint8_t> bits(S, 0);
    int any = 0;
    for (int d = 0; d < S; ++d) {
        for (int f = 0; f < 6; ++f)
            if (env->face_mask[f * S + d]) bits[d] |= (uint8_t)(1u << f);
        any |= bits[d];
    }
    const size_t fsz[6] = {(size_t)env->ny * env->nz, (size_t)env->ny * env->nz, (size_t)env->nx * env->nz,
                           (size_t)env->nx * env->nz, (size_t)env->nx * env->ny, (size_t)env->nx * env->ny};
    for (int f = 0; f < 6; ++f)
        if (!env->faces[f]) {
            BFB_CUDA(cudaMalloc(&env->faces[f], env->elem * fsz[f] * S));
            BFB_CUDA(cudaMemset(env->faces[f], 0, env->elem * fsz[f] * S));
        }
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    if (faces_host)
        for (int f = 0; f < 6; ++f) {
            int st = upload_table(env, env->faces[f], faces_host[f]);
            if (st) return st;
        }
    BFB_CUDA(cudaMemcpy(env->d_mask, bits.data(), S, cudaMemcpyHostToDevice));
    env->dir_any = any != 0;
    env->epoch++;
    return BFB_OK;
}

BFB_API int bfb_set_dirichlet(bfb_env env, const double *values, const uint8_t *activation, const uint8_t *face_mask) {
    int st = check_env(env);
    if (st) return st;
    if (!activation) return fail(BFB_ERR_INVALID_ARG, "activation must not be NULL");
    if (!values) return dirichlet_install(env, nullptr, activation, face_mask);
    const int nx = env->nx, ny = env->ny, nz = env->nz, S = env->S;
    std::vector<double> F[6];
    F[0].resize((size_t)ny * nz * S);
    F[1].resize((size_t)ny * nz * S);
    F[2].resize((size_t)nx * nz * S);
    F[3].resize((size_t)nx * nz * S);
    F[4].resize((size_t)nx * ny * S);
    F[5].resize((size_t)nx * ny * S);
    auto at = [&](int i, int j, int k, int d) { return values[(((size_t)i * ny + j) * nz + k) * S + d]; };
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
            for (int d = 0; d < S; ++d) {
                F[0][((size_t)j * nz + k) * S + d] = at(0, j, k, d);
                F[1][((size_t)j * nz + k) * S + d] = at(nx - 1, j, k, d);
            }
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k)
            for (int d = 0; d < S; ++d) {
                F[2][((size_t)i * nz + k) * S + d] = at(i, 0, k, d);
                F[3][((size_t)i * nz + k) * S + d] = at(i, ny - 1, k, d);
            }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int d = 0; d < S; ++d) {
                F[4][((size_t)i * ny + j) * S + d] = at(i, j, 0, d);
                F[5][((size_t)i * ny + j) * S + d] = at(i, j, nz - 1, d);
            }
    return dirichlet_install(env, F, activation, face_mask);
}

BFB_API int bfb_set_dirichlet_uniform(bfb_env env, const double *value_per_substrate, const uint8_t *activation,
                                      const uint8_t *face_mask) {
    int st = check_env(env);
    if (st) return st;
    if (!activation) return fail(BFB_ERR_INVALID_ARG, "activation must not be NULL");
    if (!value_per_substrate) return dirichlet_install(env, nullptr, activation, face_mask);
    const int nx = env->nx, ny = env->ny, nz = env->nz, S = env->S;
    const size_t fsz[6] = {(size_t)ny * nz, (size_t)ny * nz, (size_t)nx * nz, (size_t)nx * nz, (size_t)nx * ny,
                           (size_t)nx * ny};
    std::vector<double> F[6];
    for (int f = 0; f < 6; ++f) {
        F[f].resize(fsz[f] * S);
        for (size_t q = 0; q < fsz[f]; ++q)
            for (int d = 0; d < S; ++d) F[f][q * S + d] = value_per_substrate[d];
    }
    return dirichlet_install(env, F, activation, face_mask);
}

BFB_API int bfb_apply_dirichlet(bfb_env env) {
    int st = check_env(env);
    if (st) return st;
    st = env->precision == BFB_FP64 ? launch_dirichlet<double>(make_args<double>(env, 0, false, 0), env->stream)
                                    : launch_dirichlet<float>(make_args<float>(env, 0, false, 0), env->stream);
    return st;
}

BFB_API int bfb_diffusion_step(bfb_env env, double dt, int n_steps) {
    int st = check_env(env);
    if (st) return st;
    if (n_steps < 0) return fail(BFB_ERR_INVALID_ARG, "n_steps < 0");
    if (!(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "dt must be > 0");
    if ((st = ensure_factors(env, dt))) return st;
    return run_steps_any(env, dt, n_steps, BFB_STEP_DIFFUSION, env->stream);
}


BFB_API int bfb_set_bulk(bfb_env env, const double *supply_rate, const double *target, const double *uptake) {
    int st = check_env(env);
    if (st) return st;
    if (!supply_rate && !target && !uptake) {
        env->bulk_on = 0;
        env->epoch++;
        return BFB_OK;
    }
    if (!supply_rate || !target || !uptake) return fail(BFB_ERR_INVALID_ARG, "bulk: give all three arrays or none");
    if ((st = bulk_tabulate(env, supply_rate, target, uptake))) return st;
    env->bulk_on = 1;
    env->epoch++;
    return BFB_OK;
}

BFB_API int bfb_bulk_step(bfb_env env, double dt) {
    int st = check_env(env);
    if (st) return st;
    return run_steps_any(env, dt, 1, BFB_STEP_BULK, env->stream);
}

BFB_API int bfb_set_agents(bfb_env env, int n, const double *pos, const double *volume, const double *secretion,
                           const double *uptake, const double *saturation, const uint8_t *active, double dt) {
    int st = check_env(env);
    if (st) return st;
    if (n < 0) return fail(BFB_ERR_INVALID_ARG, "n < 0");
    if (n > 0 && (!pos || !volume || !secretion || !uptake || !saturation))
        return fail(BFB_ERR_INVALID_ARG, "agent arrays must not be NULL");
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    st = agents_build(env, n, pos, volume, secretion, uptake, saturation, active, dt);
    if (!st) {
        const size_t nS = (size_t)n * env->S;
        env->h_vol.assign(volume, volume + n);
        env->h_sec.assign(secretion, secretion + nS);
        env->h_upt.assign(uptake, uptake + nS);
        env->h_sat.assign(saturation, saturation + nS);
        env->agent_dt = dt;
    }
    env->epoch++;
    return st;
}

BFB_API int bfb_set_agent_constants(bfb_env env, int n, const int *voxel, const double *temp1, const double *temp2,
                                    const uint8_t *active) {
    int st = check_env(env);
    if (st) return st;
    if (n < 0) return fail(BFB_ERR_INVALID_ARG, "n < 0");
    if (n > 0 && (!voxel || !temp1 || !temp2)) return fail(BFB_ERR_INVALID_ARG, "agent arrays must not be NULL");
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    st = agents_build_constants(env, n, voxel, temp1, temp2, active);
    env->h_vol.clear();  // rates unknown: the adjoint gives no per-agent rate gradients
    env->h_sec.clear();
    env->h_upt.clear();
    env->h_sat.clear();
    env->epoch++;
    return st;
}

BFB_API int bfb_agent_voxels(bfb_env env, int *out) {
    int st = check_env(env);
    if (st) return st;
    if (env->n_agents == 0) return BFB_OK;
    if (!out) return fail(BFB_ERR_INVALID_ARG, "out is NULL");
    BFB_CUDA(cudaMemcpy(out, env->agent_voxel, sizeof(int) * env->n_agents, cudaMemcpyDeviceToHost));
    return BFB_OK;
}

BFB_API int bfb_cells_step(bfb_env env, double dt) {
    (void)dt;  // constants are cached by bfb_set_agents, as set_internal_uptake_constants does
    int st = check_env(env);
    if (st) return st;
    return launch_cells(env, env->stream);
}

BFB_API int bfb_simulate(bfb_env env, double dt, int n_steps, int flags) {
    int st = check_env(env);
    if (st) return st;
    if (n_steps < 0) return fail(BFB_ERR_INVALID_ARG, "n_steps < 0");
    if (!(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "dt must be > 0");
    if (flags & ~(BFB_STEP_BULK | BFB_STEP_DIFFUSION | BFB_STEP_CELLS)) return fail(BFB_ERR_INVALID_ARG, "bad flags");
    if (flags & BFB_STEP_DIFFUSION) {
        if ((st = refuse_slab(env))) return st;
        if ((st = ensure_factors(env, dt))) return st;
    }
    if (n_steps == 0) return BFB_OK;
    NvtxRange range("bfb_simulate");
    if (!env->use_graphs || env->stream == nullptr) return run_steps_any(env, dt, n_steps, flags, env->stream);
    // One step captured as a graph, replayed n_steps times.
    if (!env->graph_exec || env->graph_flags != flags || env->graph_dt != dt || env->graph_epoch != env->epoch) {
        drop_graph(env);
        cudaGraph_t graph = nullptr;
        BFB_CUDA(cudaStreamBeginCapture(env->stream, cudaStreamCaptureModeThreadLocal));
        int cst = run_steps_any(env, dt, 1, flags, env->stream);
        cudaError_t e = cudaStreamEndCapture(env->stream, &graph);
        if (cst) {
            if (graph) cudaGraphDestroy(graph);
            return cst;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&env->graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            env->graph_exec = nullptr;
            return cuda_fail(e, "cudaGraphInstantiate");
        }
        env->graph_flags = flags;
        env->graph_dt = dt;
        env->graph_epoch = env->epoch;
    }
    for (int q = 0; q < n_steps; ++q) BFB_CUDA(cudaGraphLaunch(env->graph_exec, env->stream));
    return BFB_OK;
}

BFB_API int bfb_step_host(bfb_env env, double *host_field, double dt, int n_steps) {
    int st = check_env(env);
    if (st) return st;
    if (!host_field) return fail(BFB_ERR_INVALID_ARG, "host_field is NULL");
    if ((st = refuse_slab(env))) return st;
    if ((st = ensure_factors(env, dt))) return st;
    NvtxRange range("bfb_step_host");
    cudaStream_t s = env->stream;
    if ((st = field_from_host_doubles(env, host_field, s))) return st;
    if ((st = run_steps_any(env, dt, n_steps, BFB_STEP_DIFFUSION, s))) return st;
    // a wait that ran out leaves the device field untrustworthy: report it and
    // leave the caller's host field as it was
    if ((st = env_check_device_error(env))) return st;
    if ((st = field_to_host_doubles(env, host_field, s))) return st;
    BFB_CUDA(cudaStreamSynchronize(s));
    return BFB_OK;
}

BFB_API int bfb_host_register(void *host, size_t bytes) {
    if (!host || bytes == 0) return fail(BFB_ERR_INVALID_ARG, "host is NULL or bytes is 0");
    BFB_CUDA(cudaHostRegister(host, bytes, cudaHostRegisterDefault));
    return BFB_OK;
}

BFB_API int bfb_host_unregister(void *host) {
    if (!host) return fail(BFB_ERR_INVALID_ARG, "host is NULL");
    BFB_CUDA(cudaHostUnregister(host));
    return BFB_OK;
}

// Per-phase device time, the counterpart of the reference's -DTIMING CSV
// (BioFVM_parallel.cpp:695-697, 1259-1392): events around every launch.
// ---------------------------------------------------------------------------
// Launch-shape tuning. A shape is, per axis, {TMA tiles or cp.async tiles,
// warps per CTA, row groups per TMA tile}; all shapes compute the same
// numbers. bfb_autotune times each candidate of each sweep out of place (the
// env's field -> a scratch field, so the field is unchanged) and keeps the
// fastest.
// ---------------------------------------------------------------------------
static bool tuning_valid(const int *v) {
    for (int a = 0; a < 3; ++a) {
        const int tma = v[3 * a], warps = v[3 * a + 1], chunks = v[3 * a + 2];
        if (tma < 0 || tma > 2 || warps < 1 || warps > 4 || chunks < 1 || chunks > 16) return false;
    }
    return true;
}

static void apply_tuning(bfb_env_s *env, const int *v) {
    for (int a = 0; a < 3; ++a) {
        env->tuning.tma[a] = v[3 * a];
        env->tuning.warps[a] = v[3 * a + 1];
        env->tuning.chunks[a] = v[3 * a + 2];
    }
    encode_field_maps(env);
    drop_graph(env);
    env->epoch++;
}

BFB_API int bfb_set_tuning(bfb_env env, const int *shape) {
    int st = check_env(env);
    if (st) return st;
    if (!shape) return fail(BFB_ERR_INVALID_ARG, "shape is NULL");
    if (!tuning_valid(shape)) return fail(BFB_ERR_INVALID_ARG, "tuning: tma 0..2, warps 1..4, chunks 1..16 per axis");
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    apply_tuning(env, shape);
    return BFB_OK;
}

BFB_API int bfb_get_tuning(bfb_env env, int *shape) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    if (!shape) return fail(BFB_ERR_INVALID_ARG, "shape is NULL");
    for (int a = 0; a < 3; ++a) {
        shape[3 * a] = env->tuning.tma[a];
        shape[3 * a + 1] = env->tuning.warps[a];
        shape[3 * a + 2] = env->tuning.chunks[a];
    }
    return BFB_OK;
}

}  // extern "C"

template <typename T>
static int time_candidates(bfb_env_s *env, double dt, int trials, void *scratch, int *best, double *best_ms) {
    cudaStream_t s = env->stream;
    cudaEvent_t e0, e1;
    BFB_CUDA(cudaEventCreate(&e0));
    BFB_CUDA(cudaEventCreate(&e1));
    int st = BFB_OK;
    for (int axis = 0; axis < 3 && !st; ++axis) {
        best_ms[axis] = -1.0;
        for (int tma = 1; tma >= 0 && !st; --tma)
            for (int warps : {1, 2, 4}) {
                for (int chunks : {2, 4, 8}) {
                    if (!tma && chunks != kChunks) continue;  // the cp.async tiles have a fixed stage count
                    SweepArgs<T> a = make_args<T>(env, axis, false, dt);
                    a.fo = static_cast<T *>(scratch);
                    CUtensorMap mi, mo;
                    int ci = 0, co = 0;
                    bool maps = false;
                    const int lines = strided_tile_lines(axis == 0 ? env->nx : env->ny, (int)env->elem, chunks);
                    if (axis < 2 && tma && env->use_tma)
                        maps = make_sweep_tensor_map(&mi, &ci, env->field, (int)env->elem, axis, env->nx, env->ny,
                                                     env->nz, env->S, chunks, env->Lp, lines) &&
                               make_sweep_tensor_map(&mo, &co, scratch, (int)env->elem, axis, env->nx, env->ny,
                                                     env->nz, env->S, chunks, env->Lp, lines);
                    auto launch = [&]() -> int {
                        if (axis < 2)
                            return launch_strided<T>(a, axis, axis == 0, warps, maps ? &mi : nullptr,
                                                     maps ? &mo : nullptr, ci, lines, s);
                        return launch_contig<T>(a, warps, tma && env->use_tma, s, chunks);
                    };
                    if ((st = launch())) break;  // warm
                    cudaError_t e = cudaEventRecord(e0, s);
                    for (int q = 0; q < trials && !st && e == cudaSuccess; ++q) st = launch();
                    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
                    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                    float ms = 0;
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                    if (e != cudaSuccess) st = cuda_fail(e, "autotune timing");
                    if (st) break;
                    const double per = ms / trials;
                    if (best_ms[axis] < 0 || per < best_ms[axis]) {
                        best_ms[axis] = per;
                        best[3 * axis] = tma;
                        best[3 * axis + 1] = warps;
                        best[3 * axis + 2] = tma ? chunks : env->tuning.chunks[axis];
                    }
                }
                if (st) break;
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

extern "C" {

BFB_API int bfb_autotune(bfb_env env, double dt, int trials, int *chosen, double *best_ms) {
    int st = check_env(env);
    if (st) return st;
    if (!(dt > 0) || trials < 1) return fail(BFB_ERR_INVALID_ARG, "dt must be > 0 and trials >= 1");
    if ((st = refuse_slab(env))) return st;
    if ((st = ensure_factors(env, dt))) return st;
    BFB_CUDA(cudaStreamSynchronize(env->stream));
    void *scratch = nullptr;
    BFB_CUDA(cudaMalloc(&scratch, env->elem * env->Np));
    int best[9];
    double ms[3];
    bfb_get_tuning(env, best);
    st = env->precision == BFB_FP64 ? time_candidates<double>(env, dt, trials, scratch, best, ms)
                                    : time_candidates<float>(env, dt, trials, scratch, best, ms);
    cudaFree(scratch);
    if (st) return st;
    if ((st = env_check_device_error(env))) return st;
    apply_tuning(env, best);
    if (chosen) std::copy(best, best + 9, chosen);
    if (best_ms) std::copy(ms, ms + 3, best_ms);
    return BFB_OK;
}

BFB_API int bfb_profile_steps(bfb_env env, double dt, int n_steps, int flags, double *ms_out) {
    int st = check_env(env);
    if (st) return st;
    if ((st = refuse_slab(env))) return st;
    if (!ms_out || n_steps < 1) return fail(BFB_ERR_INVALID_ARG, "ms_out NULL or n_steps < 1");
    if (!(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "dt must be > 0");
    if (flags & BFB_STEP_DIFFUSION)
        if ((st = ensure_factors(env, dt))) return st;
    for (int q = 0; q < BFB_PROFILE_PHASES; ++q) ms_out[q] = 0.0;
    cudaStream_t s = env->stream;
    cudaEvent_t ev[BFB_PROFILE_PHASES + 1];
    for (auto &e : ev) BFB_CUDA(cudaEventCreate(&e));
    static const char *const kPhaseNames[BFB_PROFILE_PHASES] = {"sweep_x", "sweep_y", "sweep_z", "bulk", "cells"};
    auto phase_ms = [&](int ph, auto &&launch) -> int {
        NvtxRange range(kPhaseNames[ph]);
        BFB_CUDA(cudaEventRecord(ev[0], s));
        int r = launch();
        if (r) return r;
        BFB_CUDA(cudaEventRecord(ev[1], s));
        BFB_CUDA(cudaEventSynchronize(ev[1]));
        float ms = 0;
        BFB_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        ms_out[ph] += ms;
        return BFB_OK;
    };
    for (int q = 0; q < n_steps && !st; ++q) {
        const bool fp64 = env->precision == BFB_FP64;
        if (flags & BFB_STEP_DIFFUSION) {
            const bool bulk = (flags & BFB_STEP_BULK) != 0;
            st = phase_ms(0, [&] {
                return fp64 ? launch_strided_env<double>(env, 0, bulk, dt, s)
                            : launch_strided_env<float>(env, 0, bulk, dt, s);
            });
            if (!st)
                st = phase_ms(1, [&] {
                    return fp64 ? launch_strided_env<double>(env, 1, false, dt, s)
                                : launch_strided_env<float>(env, 1, false, dt, s);
                });
            if (!st)
                st = phase_ms(2, [&] {
                    const bool tz = env->use_tma != 0 && env->tuning.tma[2] != 0;
                    return fp64 ? launch_contig<double>(make_args<double>(env, 2, false, dt), env->tuning.warps[2], tz,
                                                        s, env->tuning.chunks[2])
                                : launch_contig<float>(make_args<float>(env, 2, false, dt), env->tuning.warps[2], tz, s,
                                                       env->tuning.chunks[2]);
                });
        } else if (flags & BFB_STEP_BULK) {
            st = phase_ms(3, [&] {
                return fp64 ? launch_bulk<double>(make_args<double>(env, 0, true, dt), env->Np, s)
                            : launch_bulk<float>(make_args<float>(env, 0, true, dt), env->Np, s);
            });
        }
        if (!st && (flags & BFB_STEP_CELLS)) st = phase_ms(4, [&] { return launch_cells(env, s); });
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return st;
}

BFB_API int bfb_checksum(bfb_env env, double *out) {
    int st = check_env(env);
    if (st) return st;
    if (!out) return fail(BFB_ERR_INVALID_ARG, "out is NULL");
    if ((st = checksum_prepare(env))) return st;
    double *dout = env->partials + (size_t)env->partial_blocks * env->S;
    if ((st = launch_checksum(env, dout, env->stream))) return st;
    BFB_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * env->S, cudaMemcpyDeviceToHost, env->stream));
    return env_check_device_error(env);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// x-slab decomposition (BioFVM_parallel.cpp:108-144 splits the x planes over
// ranks; :832-873 and :948-1255 pipeline the x lines' Thomas solve across
// them). A slab env is an ordinary env of nx_local planes whose x factor
// tables are those of the whole line of nx_global planes; its x sweep runs in
// the two halves below, the y and z sweeps are its own.
// ---------------------------------------------------------------------------
BFB_API int bfb_create_slab(bfb_env *out, int nx_global, int x0, int nx_local, int ny, int nz, int n_substrates,
                            double dx, int device) {
    if (!out) return fail(BFB_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (nx_global < 2 || x0 < 0 || nx_local < 1 || (long long)x0 + nx_local > nx_global)
        return fail(BFB_ERR_SIZE, "a slab needs nx_global >= 2 and 0 <= x0 < x0 + nx_local <= nx_global");
    int st = bfb_create(out, nx_local, ny, nz, n_substrates, dx, BFB_FP64, device);
    if (st) return st;
    bfb_env_s *env = *out;
    env->nx_global = nx_global;
    env->x0 = x0;
    env->bbox[0] = x0 * dx;
    env->bbox[3] = (x0 + nx_local) * dx;
    // the x factor tables hold the whole line
    cudaFree(env->fac_tab[0]);
    cudaFree(env->fac_head[0]);
    env->fac_tab[0] = env->fac_head[0] = nullptr;
    cudaError_t e = cudaMalloc(&env->fac_tab[0], env->elem * 4 * (size_t)nx_global * n_substrates);
    if (e == cudaSuccess)
        e = cudaMalloc(&env->fac_head[0], env->elem * 4 * (size_t)n_substrates * ((nx_global + 3) / 4 * 4));
    if (e != cudaSuccess) {
        bfb_destroy(env);
        *out = nullptr;
        return cuda_fail(e, "cudaMalloc");
    }
    return BFB_OK;
}

BFB_API int bfb_slab_info(bfb_env env, int *nx_global, int *x0, long long *lines) {
    int st = check_env(env);
    if (st) return st;
    if (nx_global) *nx_global = env->nx_global ? env->nx_global : env->nx;
    if (x0) *x0 = env->x0;
    if (lines) *lines = (long long)env->ny * env->Lp;
    return BFB_OK;
}

static int slab_half_args(bfb_env_s *env, double dt, long long line0, long long line1) {
    if (!env->nx_global) return fail(BFB_ERR_STATE, "not an x-slab env (bfb_create_slab)");
    if (!(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "dt must be > 0");
    if (line0 < 0 || line1 < line0 || line1 > (long long)env->ny * env->Lp)
        return fail(BFB_ERR_INVALID_ARG, "line range outside [0, ny * pitch]");
    return ensure_factors(env, dt);
}

BFB_API int bfb_slab_x_forward(bfb_env env, double dt, const double *prev_in, double *prev_out, long long line0,
                               long long line1) {
    int st = check_env(env);
    if (st) return st;
    if ((st = slab_half_args(env, dt, line0, line1))) return st;
    if (env->x0 > 0 && !prev_in) return fail(BFB_ERR_INVALID_ARG, "prev_in is NULL past the grid's first plane");
    NvtxRange range("bfb_slab_x_forward");
    return launch_slab_x_forward(make_args<double>(env, 0, false, dt), env->x0, env->nx_global, line0, line1,
                                 env->x0 > 0 ? prev_in : nullptr, prev_out, env->stream);
}

BFB_API int bfb_slab_x_backward(bfb_env env, double dt, const double *next_in, double *next_out, long long line0,
                                long long line1) {
    int st = check_env(env);
    if (st) return st;
    if ((st = slab_half_args(env, dt, line0, line1))) return st;
    const bool last = env->x0 + env->nx == env->nx_global;
    if (!last && !next_in) return fail(BFB_ERR_INVALID_ARG, "next_in is NULL before the grid's last plane");
    NvtxRange range("bfb_slab_x_backward");
    return launch_slab_x_backward(make_args<double>(env, 0, false, dt), env->x0, env->nx_global, line0, line1,
                                  last ? nullptr : next_in, next_out, env->stream);
}

BFB_API int bfb_slab_yz(bfb_env env, double dt) {
    int st = check_env(env);
    if (st) return st;
    if ((st = slab_half_args(env, dt, 0, 0))) return st;
    NvtxRange range("bfb_slab_yz");
    if ((st = launch_strided_env<double>(env, 1, false, dt, env->stream))) return st;
    return launch_contig<double>(make_args<double>(env, 2, false, dt), env->tuning.warps[2],
                                 env->use_tma != 0 && env->tuning.tma[2] != 0, env->stream, env->tuning.chunks[2]);
}
