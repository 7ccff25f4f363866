// bfb_slab.cu -- the x sweep of one x-slab of a larger grid, in two halves.
//
// The reference splits the grid's x axis over MPI ranks
// (BioFVM_parallel.cpp:108-144); its x lines then cross rank boundaries, and
// it solves them with a pipelined exchange: the forward elimination of rank r
// starts from the last forward value that rank r-1 sends for each line, and
// the back substitution of rank r starts from the first back-substituted value
// that rank r+1 sends (BioFVM_parallel.cpp:948-1255, send/receive at
// :832-873). Here one slab env holds x planes [x0, x0 + nx) of a grid of
// nx_global planes, with the Thomas factors of the whole line; its forward
// half stores the forward values in place and gives the last one per line,
// its backward half takes the neighbour's value and finishes the lines. Each
// line's operations and their order are those of the whole-grid sweep, so
// the slabs together reproduce it bit for bit (FP64).
//
// One thread per x line: the lines of a slab are its ny * Lp columns, so a
// warp's loads and stores of one row are 32 consecutive elements. The line
// range [line0, line1) lets the caller pipeline chunks of lines across ranks.
#include "bfb_line.cuh"

namespace bfb {

namespace {

// Rows whose loads are in flight together, per half (measured at 256^3 x 8,
// one slab: forward 4 rows 0.379 ms, 8 rows 0.747, 16 rows 0.881; backward
// 16 rows 0.378 ms, 4 rows 0.436). The forward's four-operation chain per row
// gains nothing from deeper blocks and loses occupancy to their registers.
constexpr int kSlabFwdBlock = 4;
constexpr int kSlabBwdBlock = 16;

struct SlabColumn {
    int cj, ck, d;
    bool real;
};

__device__ __forceinline__ SlabColumn slab_column(const SweepArgs<double> &a, long long cl) {
    SlabColumn c;
    c.cj = (int)(cl / a.Lp);
    const int q = (int)(cl - (long long)c.cj * a.Lp);
    c.real = q < a.nz * a.S;  // padding columns of a padded row hold no field value
    c.ck = q / a.S;
    c.d = q - c.ck * a.S;
    return c;
}

__global__ void __launch_bounds__(256) slab_x_forward_kernel(SweepArgs<double> a, int x0, int nglob, long long line0,
                                                              long long line1, const double *__restrict__ prev_in,
                                                              double *__restrict__ prev_out) {
    const long long cl = line0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cl >= line1) return;
    const SlabColumn c = slab_column(a, cl);
    if (!c.real) return;
    const int nloc = a.nx;
    const long long P = (long long)a.ny * a.Lp;
    const unsigned m = a.dir.any ? a.dir.mask[c.d] : 0u;
    // the env's x-face bits are set only where the slab holds the grid's face
    const bool lo_dir = (m & 1u) && x0 == 0, hi_dir = (m & 2u) && x0 + nloc == nglob;
    double *f = a.f + cl;
    auto xin = [&](int r) -> double {  // input row after the step's leading Dirichlet
        double x = f[(size_t)r * P];
        if ((lo_dir && x0 + r == 0) || (hi_dir && x0 + r == nglob - 1)) x = dir_value(a.dir, r, c.cj, c.ck, c.d);
        return x;
    };
    LineSolver<double> L(a, c.d);
    int r = 0;
    if (x0 == 0) {
        f[0] = L.first(xin(0), 0.0);
        r = 1;
    } else {
        L.prev = prev_in[cl];
    }
    // rows in blocks: a block's loads are issued before its stores (a store
    // may alias a later row, so the compiler keeps program order), so the
    // loads of a block are in flight together
    for (; r + kSlabFwdBlock <= nloc; r += kSlabFwdBlock) {
        double v[kSlabFwdBlock];
#pragma unroll
        for (int u = 0; u < kSlabFwdBlock; ++u) v[u] = xin(r + u);
#pragma unroll
        for (int u = 0; u < kSlabFwdBlock; ++u) v[u] = L.fwd<false>(v[u], x0 + r + u);
#pragma unroll
        for (int u = 0; u < kSlabFwdBlock; ++u) f[(size_t)(r + u) * P] = v[u];
    }
    for (; r < nloc; ++r) f[(size_t)r * P] = L.fwd<false>(xin(r), x0 + r);
    if (prev_out) prev_out[cl] = L.prev;
}

__global__ void __launch_bounds__(256) slab_x_backward_kernel(SweepArgs<double> a, int x0, int nglob, long long line0,
                                                               long long line1, const double *__restrict__ next_in,
                                                               double *__restrict__ next_out) {
    const long long cl = line0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cl >= line1) return;
    const SlabColumn c = slab_column(a, cl);
    if (!c.real) return;
    const int nloc = a.nx;
    const long long P = (long long)a.ny * a.Lp;
    const unsigned m = a.dir.any ? a.dir.mask[c.d] : 0u;
    const bool lo_dir = (m & 1u) && x0 == 0, hi_dir = (m & 2u) && x0 + nloc == nglob;
    // the whole line lies on an active y or z face
    const bool col_dir = ((m & 4u) && c.cj == 0) || ((m & 8u) && c.cj == a.ny - 1) || ((m & 16u) && c.ck == 0) ||
                         ((m & 32u) && c.ck == a.nz - 1);
    double *f = a.f + cl;
    LineSolver<double> L(a, c.d);
    int r = nloc - 1;
    if (x0 + nloc == nglob) {  // the grid's last row starts the back substitution with its forward value
        L.prev = f[(size_t)r * P];
        double y = L.out_last();
        if (hi_dir || col_dir) y = dir_value(a.dir, r, c.cj, c.ck, c.d);
        f[(size_t)r * P] = y;
        --r;
    } else {
        L.next = next_in[cl];
    }
    auto out = [&](int q, double y) -> double {  // the stored value; the recurrence carries y
        return ((lo_dir && x0 + q == 0) || col_dir) ? dir_value(a.dir, q, c.cj, c.ck, c.d) : y;
    };
    for (; r - kSlabBwdBlock + 1 >= 0; r -= kSlabBwdBlock) {
        double v[kSlabBwdBlock];
#pragma unroll
        for (int u = 0; u < kSlabBwdBlock; ++u) v[u] = f[(size_t)(r - u) * P];
#pragma unroll
        for (int u = 0; u < kSlabBwdBlock; ++u) v[u] = L.bwd<false>(v[u], x0 + r - u);
#pragma unroll
        for (int u = 0; u < kSlabBwdBlock; ++u) f[(size_t)(r - u) * P] = out(r - u, v[u]);
    }
    for (; r >= 0; --r) f[(size_t)r * P] = out(r, L.bwd<false>(f[(size_t)r * P], x0 + r));
    if (next_out) next_out[cl] = L.next;
}

}  // namespace

int launch_slab_x_forward(const SweepArgs<double> &a, int x0, int nglob, long long line0, long long line1,
                          const double *prev_in, double *prev_out, cudaStream_t s) {
    if (line1 <= line0) return BFB_OK;
    const long long n = line1 - line0;
    slab_x_forward_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, x0, nglob, line0, line1, prev_in, prev_out);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

int launch_slab_x_backward(const SweepArgs<double> &a, int x0, int nglob, long long line0, long long line1,
                           const double *next_in, double *next_out, cudaStream_t s) {
    if (line1 <= line0) return BFB_OK;
    const long long n = line1 - line0;
    slab_x_backward_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, x0, nglob, line0, line1, next_in, next_out);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

}  // namespace bfb
