// bfb_line.cuh -- device helpers shared by the sweep kernels: async copies,
// Dirichlet lookups, the bulk update, the FP64 division and the per-lane
// Thomas recurrences.
#pragma once
#include "bfb_sweeps.cuh"

namespace bfb {

constexpr int kMaxSmem = 227 * 1024;  // opt-in dynamic shared memory per CTA on sm_100a

// ---------------------------------------------------------------------------
// cp.async helpers (LDGSTS: global -> shared without staging in registers)
// ---------------------------------------------------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_wait_dyn(int pending) {
    switch (pending) {
    case 0: cp_wait<0>(); break;
    case 1: cp_wait<1>(); break;
    case 2: cp_wait<2>(); break;
    default: cp_wait<3>(); break;
    }
}

// ---------------------------------------------------------------------------
// Dirichlet lookups
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T dir_value(const DirFaces<T> &F, int i, int j, int k, int d) {
    if (i == 0) return F.face[0][((size_t)j * F.nz + k) * F.S + d];
    if (i == F.nx - 1) return F.face[1][((size_t)j * F.nz + k) * F.S + d];
    if (j == 0) return F.face[2][((size_t)i * F.nz + k) * F.S + d];
    if (j == F.ny - 1) return F.face[3][((size_t)i * F.nz + k) * F.S + d];
    if (k == 0) return F.face[4][((size_t)i * F.ny + j) * F.S + d];
    return F.face[5][((size_t)i * F.ny + j) * F.S + d];
}

__device__ __forceinline__ bool on_active_face(unsigned m, int i, int j, int k, int nx, int ny, int nz) {
    return ((m & 1u) && i == 0) || ((m & 2u) && i == nx - 1) || ((m & 4u) && j == 0) ||
           ((m & 8u) && j == ny - 1) || ((m & 16u) && k == 0) || ((m & 32u) && k == nz - 1);
}

// ---------------------------------------------------------------------------
// Bulk source/sink update (BioFVM_microenvironment.cpp:1131-1148):
//   rho = (rho + dt*A) / ((B*dt) + 1) with A = S*T, B = U + S; the first
//   product is fused as in the reference build.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double bulk_update(double r, double A, double B, double dt) {
    return __ddiv_rn(__fma_rn(dt, A, r), __dadd_rn(__dmul_rn(B, dt), 1.0));
}
__device__ __forceinline__ float bulk_update(float r, float A, float B, float dt) {
    return __fdiv_rn(__fmaf_rn(dt, A, r), __fmaf_rn(B, dt, 1.0f));
}

// ---------------------------------------------------------------------------
// Correctly rounded t/b from r = RN(1/b), by one residual correction
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990):
//   q0 = RN(t*r), e = t - b*q0 (exact by FMA), q = RN(q0 + e*r) = RN(t/b).
// Three dependent FP64 operations instead of the IEEE division sequence,
// which on sm_100a costs ~13x more per dependent step (measured). The FP64
// parity tests check the results bit for bit against IEEE division; the
// argument needs t and e normal (|t| well above 2^-969), which field values
// of any physical run are.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double div_rcp(double t, double b, double r) {
    const double q0 = __dmul_rn(t, r);
    const double e = __fma_rn(-q0, b, t);
    return __fma_rn(e, r, q0);
}

// ---------------------------------------------------------------------------
// Lean per-lane recurrences for the shared-memory kernels. fwd<TAIL> /
// bwd<TAIL> read the factor tables only when TAIL is false (rows < m0 and the
// last row); TAIL rows use the register copies.
// ---------------------------------------------------------------------------
template <typename T>
struct LineSolver;

template <>
struct LineSolver<double> {
    const double *den, *cb, *rcp;
    double den_t, cb_t, rcp_t, c1;
    int S;
    double prev, next;
    __device__ __forceinline__ LineSolver(const SweepArgs<double> &a, int d) {
        den = a.fac.t0 + d;
        cb = a.fac.t1 + d;
        rcp = a.fac.t2 + d;
        den_t = a.fac.tail[d];
        cb_t = a.fac.tail[a.S + d];
        rcp_t = a.fac.tail[2 * a.S + d];
        c1 = a.c1[d];
        S = a.S;
    }
    // returns the value stored for the backward pass (xref: FP32 only)
    __device__ __forceinline__ double first(double x0, double) {
        prev = div_rcp(x0, den[0], rcp[0]);
        return prev;
    }
    template <bool TAIL>
    __device__ __forceinline__ double fwd(double x, int r) {
        const double t = __fma_rn(c1, prev, x);
        if (TAIL) {
            prev = div_rcp(t, den_t, rcp_t);
        } else {
            const size_t q = (size_t)r * S;
            prev = div_rcp(t, den[q], rcp[q]);
        }
        return prev;
    }
    __device__ __forceinline__ double out_last() {
        next = prev;
        return next;
    }
    template <bool TAIL>
    __device__ __forceinline__ double bwd(double z, int r) {
        next = __fma_rn(-(TAIL ? cb_t : cb[(size_t)r * S]), next, z);
        return next;
    }
};

template <>
struct LineSolver<float> {
    const float *rh, *rl, *a, *cb;
    float rh_t, rl_t, a_t, cb_t, gh, gl;
    int S;
    float xb, p, next;
    __device__ __forceinline__ LineSolver(const SweepArgs<float> &A, int d) {
        rh = A.fac.t0 + d;
        rl = A.fac.t1 + d;
        a = A.fac.t2 + d;
        cb = A.fac.t3 + d;
        rh_t = A.fac.tail[d];
        rl_t = A.fac.tail[A.S + d];
        a_t = A.fac.tail[2 * A.S + d];
        cb_t = A.fac.tail[3 * A.S + d];
        gh = A.g[d];
        gl = A.g[A.S + d];
        S = A.S;
    }
    // xref is the deviation reference: the line's row 1 (row 0 when n == 1).
    // Not row 0, which on a Dirichlet line is the boundary value and can be
    // far from the interior.
    __device__ __forceinline__ float first(float x0, float xref) {
        xb = xref;
        const float dlt = __fsub_rn(x0, xb);
        p = __fmaf_rn(dlt, rh[0], __fmul_rn(dlt, rl[0]));
        return p;
    }
    template <bool TAIL>
    __device__ __forceinline__ float fwd(float x, int r) {
        const float dlt = __fsub_rn(x, xb);
        if (TAIL) {
            p = __fmaf_rn(a_t, p, __fmaf_rn(dlt, rh_t, __fmul_rn(dlt, rl_t)));
        } else {
            const size_t q = (size_t)r * S;
            p = __fmaf_rn(a[q], p, __fmaf_rn(dlt, rh[q], __fmul_rn(dlt, rl[q])));
        }
        return p;
    }
    __device__ __forceinline__ float y(float v) const { return __fmaf_rn(xb, gh, __fmaf_rn(xb, gl, v)); }
    __device__ __forceinline__ float out_last() {
        next = p;
        return y(next);
    }
    template <bool TAIL>
    __device__ __forceinline__ float bwd(float z, int r) {
        next = __fmaf_rn(-(TAIL ? cb_t : cb[(size_t)r * S]), next, z);
        return y(next);
    }
};

}  // namespace bfb
