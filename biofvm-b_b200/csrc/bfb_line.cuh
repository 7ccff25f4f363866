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
// the same with the shared-memory address already in the shared window
template <int BYTES>
__device__ __forceinline__ void cp_async_s(unsigned s, const void *gmem) {
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

// Four consecutive entries (16-byte aligned) of a head table row block.
__device__ __forceinline__ void load4(const float *p, float (&v)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
}
__device__ __forceinline__ void load4(const double *p, double (&v)[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}

// ---------------------------------------------------------------------------
// Lean per-lane recurrences for the shared-memory kernels. fwd<TAIL> /
// bwd<TAIL> read the factor tables only when TAIL is false (rows < m0 and the
// last row); TAIL rows use the register copies.
// ---------------------------------------------------------------------------
template <typename T>
struct LineSolver;

// Head rows (rows below m0, whose factors vary by row) of a line, with the
// factors read four rows at a time from the head tables; the operations are
// those of fwd<false> / bwd<false>. ld(q) reads row q's value, st(q, v)
// writes it. head_forward covers rows [r, end) and returns end;
// head_backward covers rows r, r-1, ..., stop and returns stop - 1, calling
// st for those rows in that order.
template <typename T, typename LD, typename ST>
__device__ __forceinline__ int head_forward(LineSolver<T> &L, int r, int end, LD ld, ST st) {
    int q = r;
    for (; q < end && (q & 3); ++q) st(q, L.fwd_row(ld(q), q));
    for (; q + 4 <= end; q += 4) {
        typename LineSolver<T>::Quad f;
        L.fwd_quad(q, f);
#pragma unroll
        for (int u = 0; u < 4; ++u) st(q + u, L.fwd_q(ld(q + u), f, u));
    }
    for (; q < end; ++q) st(q, L.fwd_row(ld(q), q));
    return q;
}
// Tail rows (factors in registers) in blocks of kTailBlock: a block's
// inputs are read first, the work off the recurrence (tpre / bpost) is done
// for the whole block, and only the one-operation recurrence (tstep /
// bstep) runs row after row; the operations are those of fwd<true> /
// bwd<true>. ld(q) reads row q's input, st(q, v) writes its output.
// tail_forward covers rows [r, end) and returns end; tail_backward covers
// rows r, r-1, ..., stop and returns stop - 1, calling st for those rows in
// that order (callers may rely on it).
constexpr int kTailBlock = 24;  // measured: 4 < 8 < 16 < 24 > 32 at 256^3 x 8
template <typename T, typename LD, typename ST>
__device__ __forceinline__ int tail_forward(LineSolver<T> &L, int r, int end, LD ld, ST st) {
    for (; r + kTailBlock <= end; r += kTailBlock) {
        T v[kTailBlock];
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) v[u] = ld(r + u);
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) v[u] = L.tpre(v[u]);
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) v[u] = L.tstep(v[u]);
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) st(r + u, v[u]);
    }
    for (; r < end; ++r) st(r, L.tstep(L.tpre(ld(r))));
    return r;
}
template <typename T, typename LD, typename ST>
__device__ __forceinline__ int tail_backward(LineSolver<T> &L, int r, int stop, LD ld, ST st) {
    for (; r - kTailBlock + 1 >= stop; r -= kTailBlock) {
        T v[kTailBlock];
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) v[u] = ld(r - u);
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) v[u] = L.bstep(v[u]);
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) v[u] = L.bpost(v[u]);
#pragma unroll
        for (int u = 0; u < kTailBlock; ++u) st(r - u, v[u]);
    }
    for (; r >= stop; --r) st(r, L.bpost(L.bstep(ld(r))));
    return r;
}

template <typename T, typename LD, typename ST>
__device__ __forceinline__ int head_backward(LineSolver<T> &L, int r, int stop, LD ld, ST st) {
    int q = r;
    for (; q >= stop && ((q + 1) & 3); --q) st(q, L.bwd_c(ld(q), L.hd[L.hk_cb + q]));
    for (; q - 3 >= stop; q -= 4) {
        T c[4];
        load4(L.hd + L.hk_cb + q - 3, c);
#pragma unroll
        for (int u = 0; u < 4; ++u) st(q - u, L.bwd_c(ld(q - u), c[3 - u]));
    }
    for (; q >= stop; --q) st(q, L.bwd_c(ld(q), L.hd[L.hk_cb + q]));
    return q;
}

template <>
struct LineSolver<double> {
    const double *den, *cb, *rcp;
    const double *hd;  // head tables of this lane's substrate: den at 0, cb at hk_cb, rcp at 2*hk_cb
    int hk_cb;
    double den_t, cb_t, rcp_t, c1;
    int S;
    double prev, next;
    __device__ __forceinline__ LineSolver(const SweepArgs<double> &a, int d) {
        den = a.fac.t0 + d;
        cb = a.fac.t1 + d;
        rcp = a.fac.t2 + d;
        hd = a.fac.head + (size_t)d * a.fac.hpad;
        hk_cb = a.S * a.fac.hpad;
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
    // head rows from the head tables (head_forward / head_backward)
    struct Quad {
        double den[4], rcp[4];
    };
    __device__ __forceinline__ void fwd_quad(int q, Quad &f) const {
        load4(hd + q, f.den);
        load4(hd + 2 * hk_cb + q, f.rcp);
    }
    __device__ __forceinline__ double fwd_q(double x, const Quad &f, int u) {
        prev = div_rcp(__fma_rn(c1, prev, x), f.den[u], f.rcp[u]);
        return prev;
    }
    __device__ __forceinline__ double fwd_row(double x, int q) {
        prev = div_rcp(__fma_rn(c1, prev, x), hd[q], hd[2 * hk_cb + q]);
        return prev;
    }
    __device__ __forceinline__ double bwd_c(double z, double c) {
        next = __fma_rn(-c, next, z);
        return next;
    }
    // tail rows split for tail_forward / tail_backward (all of FP64's work is on the recurrence)
    __device__ __forceinline__ double tpre(double x) const { return x; }
    __device__ __forceinline__ double tstep(double x) {
        prev = div_rcp(__fma_rn(c1, prev, x), den_t, rcp_t);
        return prev;
    }
    __device__ __forceinline__ double bstep(double z) {
        next = __fma_rn(-cb_t, next, z);
        return next;
    }
    __device__ __forceinline__ double bpost(double v) const { return v; }
};

template <>
struct LineSolver<float> {
    const float *rh, *rl, *a, *cb;
    const float *hd;  // head tables of this lane's substrate: rh, rl, a, cb at k*hk_cb, k = 0..3
    int hk, hk_cb;    // offsets of the rl and cb tables
    float rh_t, rl_t, a_t, cb_t, gh, gl;
    int S;
    float xb, p, next;
    __device__ __forceinline__ LineSolver(const SweepArgs<float> &A, int d) {
        rh = A.fac.t0 + d;
        rl = A.fac.t1 + d;
        a = A.fac.t2 + d;
        cb = A.fac.t3 + d;
        hd = A.fac.head + (size_t)d * A.fac.hpad;
        hk = A.S * A.fac.hpad;
        hk_cb = 3 * hk;
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
    // head rows from the head tables (head_forward / head_backward)
    struct Quad {
        float rh[4], rl[4], a[4];
    };
    __device__ __forceinline__ void fwd_quad(int q, Quad &f) const {
        load4(hd + q, f.rh);
        load4(hd + hk + q, f.rl);
        load4(hd + 2 * hk + q, f.a);
    }
    __device__ __forceinline__ float fwd_q(float x, const Quad &f, int u) {
        const float dlt = __fsub_rn(x, xb);
        p = __fmaf_rn(f.a[u], p, __fmaf_rn(dlt, f.rh[u], __fmul_rn(dlt, f.rl[u])));
        return p;
    }
    __device__ __forceinline__ float fwd_row(float x, int q) {
        const float dlt = __fsub_rn(x, xb);
        p = __fmaf_rn(hd[2 * hk + q], p, __fmaf_rn(dlt, hd[q], __fmul_rn(dlt, hd[hk + q])));
        return p;
    }
    __device__ __forceinline__ float bwd_c(float z, float c) {
        next = __fmaf_rn(-c, next, z);
        return y(next);
    }
    // tail rows split for tail_forward / tail_backward
    __device__ __forceinline__ float tpre(float x) const {
        const float dlt = __fsub_rn(x, xb);
        return __fmaf_rn(dlt, rh_t, __fmul_rn(dlt, rl_t));
    }
    __device__ __forceinline__ float tstep(float w) {
        p = __fmaf_rn(a_t, p, w);
        return p;
    }
    __device__ __forceinline__ float bstep(float z) {
        next = __fmaf_rn(-cb_t, next, z);
        return next;
    }
    __device__ __forceinline__ float bpost(float v) const { return y(v); }
};

}  // namespace bfb
