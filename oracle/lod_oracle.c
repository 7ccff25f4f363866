/*
 * lod_oracle.c -- CPU restatement of BioFVM-B's diffusion-decay hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the CUDA product is checked
 * against. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg load it. Parity pinned bit-for-bit against the reference library built
 * from its own sources (oracle/_ref) and against tests/golden/.
 *
 * Floating-point contraction. The reference is built by g++ in C++ mode with
 * -march=native and no -ffp-contract flag (reference Makefile:45), and g++'s
 * C++ default is -ffp-contract=fast: every `y += a*b` / `y -= a*b` on the path
 * becomes one fused multiply-add on any FMA-capable CPU, and the AVX256D
 * solver spells the same FMAs out with intrinsics (BioFVM_parallel.cpp:
 * 1715-1735, 1829-1867). This file is compiled with -ffp-contract=off and
 * writes those fused operations as explicit fma() calls (correctly rounded),
 * so its results equal the reference's bit for bit, and equal nothing else
 * by accident. Each function cites the reference lines whose arithmetic it
 * restates, in the same operation order.
 */
#include "lod_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* BioFVM_parallel.cpp:780-788: thomas_constant1 = D; *= dt; /= dx; /= dx. */
void orc_constant1(int S, double dt, double dx, const double *D, double *c1)
{
    for (int d = 0; d < S; ++d) {
        double v = D[d] * dt;
        v /= dx;
        v /= dx;
        c1[d] = v;
    }
}

/* BioFVM_parallel.cpp:780-912 for one axis of length n (single rank):
 *   c1 = dt*D/dx^2, c2 = dt*lambda/3, c3 = 1 + c1 + c1 + c2, c3a = 1 + c1 + c2
 *   c[] = -c1, denom[] = c3, denom[0] = denom[n-1] = c3a (n == 1: 1 + c2)
 *   c[0] /= denom[0]; for m >= 1: denom[m] += c1*c[m-1] (axpy, fused);
 *   c[m] /= denom[m]. */
void orc_factors(int n, int S, double dt, double dx, const double *D, const double *lambda,
                 double *denom, double *c)
{
    for (int d = 0; d < S; ++d) {
        double c1 = D[d] * dt;
        c1 /= dx;
        c1 /= dx;
        double c2 = lambda[d] * dt;
        c2 /= 3.0;
        double c3 = 1.0;
        c3 += c1;
        c3 += c1;
        c3 += c2;
        double c3a = 1.0;
        c3a += c1;
        c3a += c2;
        for (int m = 0; m < n; ++m) {
            c[(size_t)m * S + d] = -c1;
            denom[(size_t)m * S + d] = c3;
        }
        denom[d] = c3a;
        denom[(size_t)(n - 1) * S + d] = c3a;
        if (n == 1) {
            double t = 1.0;
            t += c2;
            denom[d] = t;
        }
        c[d] /= denom[d];
        for (int m = 1; m < n; ++m) {
            denom[(size_t)m * S + d] = fma(c1, c[(size_t)(m - 1) * S + d], denom[(size_t)m * S + d]);
            c[(size_t)m * S + d] /= denom[(size_t)m * S + d];
        }
    }
}

static inline int on_face(int f, int i, int j, int k, int nx, int ny, int nz)
{
    switch (f) {
    case 0: return i == 0;
    case 1: return i == nx - 1;
    case 2: return j == 0;
    case 3: return j == ny - 1;
    case 4: return k == 0;
    default: return k == nz - 1;
    }
}

/* BioFVM_microenvironment.cpp:381-484: overwrite every outer-face voxel of
 * each active substrate with its stored Dirichlet value. */
void orc_dirichlet(double *rho, int nx, int ny, int nz, int S, const double *values,
                   const uint8_t *face_mask)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int face = i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1;
                if (!face) continue;
                size_t base = (((size_t)i * ny + j) * nz + k) * S;
                for (int d = 0; d < S; ++d) {
                    int act = 0;
                    for (int f = 0; f < 6 && !act; ++f)
                        act = face_mask[f * S + d] && on_face(f, i, j, k, nx, ny, nz);
                    if (act) rho[base + d] = values[base + d];
                }
            }
}

/* One line of a Thomas sweep: forward elimination then back substitution
 * (x: BioFVM_parallel.cpp:948-978, 1129-1148; y: 1274-1317; z: 1334-1378):
 *   u[0] /= den[0]; u[m] = fma(c1, u[m-1], u[m]) / den[m];
 *   u[m] = fma(-c[m], u[m+1], u[m]) for m = n-2 .. 0. */
static void thomas_line(double *rho, size_t start, size_t stride, int n, int S, int d,
                        const double *den, const double *c, double c1)
{
    size_t idx = start;
    rho[idx] /= den[d];
    for (int m = 1; m < n; ++m) {
        size_t nxt = idx + stride;
        rho[nxt] = fma(c1, rho[idx], rho[nxt]);
        rho[nxt] /= den[(size_t)m * S + d];
        idx = nxt;
    }
    for (int m = n - 2; m >= 0; --m) {
        size_t prv = idx - stride;
        rho[prv] = fma(-c[(size_t)m * S + d], rho[idx], rho[prv]);
        idx = prv;
    }
}

void orc_lod_step(double *rho, int nx, int ny, int nz, int S,
                  const double *denx, const double *cx, const double *deny, const double *cy,
                  const double *denz, const double *cz, const double *c1,
                  const double *dir_values, const uint8_t *face_mask)
{
    size_t ij = (size_t)ny * nz * S, jj = (size_t)nz * S, kj = (size_t)S;
    orc_dirichlet(rho, nx, ny, nz, S, dir_values, face_mask);
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
            for (int d = 0; d < S; ++d)
                thomas_line(rho, j * jj + k * kj + d, ij, nx, S, d, denx, cx, c1[d]);
    orc_dirichlet(rho, nx, ny, nz, S, dir_values, face_mask);
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k)
            for (int d = 0; d < S; ++d)
                thomas_line(rho, i * ij + k * kj + d, jj, ny, S, d, deny, cy, c1[d]);
    orc_dirichlet(rho, nx, ny, nz, S, dir_values, face_mask);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int d = 0; d < S; ++d)
                thomas_line(rho, i * ij + j * jj + d, kj, nz, S, d, denz, cz, c1[d]);
    orc_dirichlet(rho, nx, ny, nz, S, dir_values, face_mask);
}

/* BioFVM_microenvironment.cpp:1122-1148: temp2 = T*S; rho += dt*temp2 (fused);
 * temp3 = ((U + S)*dt) + 1; rho /= temp3. */
void orc_bulk_step(double *rho, int64_t V, int S, double dt, const double *S_rate,
                   const double *T_target, const double *U_rate)
{
    for (int64_t v = 0; v < V; ++v)
        for (int d = 0; d < S; ++d) {
            size_t e = (size_t)v * S + d;
            double st = T_target[e] * S_rate[e];
            rho[e] = fma(dt, st, rho[e]);
            double t3 = U_rate[e] + S_rate[e];
            t3 *= dt;
            t3 += 1.0;
            rho[e] /= t3;
        }
}

/* C's (int) conversion of a double truncates toward zero, as the reference's
 * (int) casts do (BioFVM_parallel.cpp:434-446). */
static int clamp_axis(double p, double lo, double hi, double h)
{
    int v = (int)floor((p - lo) / h);
    int g = (int)((hi - lo) / h);
    if (v >= g) v = g - 1;
    if (v < 0) v = 0;
    return v;
}

void orc_bin_agents(int n, const double *pos, const double *bbox, double dx, double dy, double dz,
                    int nx, int ny, int nz, int *out_voxel)
{
    int V = nx * ny * nz;
    for (int a = 0; a < n; ++a) {
        double x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
        if (x < bbox[0] || x > bbox[3] || y < bbox[1] || y > bbox[4] || z < bbox[2] || z > bbox[5]) {
            out_voxel[a] = -1;
            continue;
        }
        int xi = clamp_axis(x, bbox[0], bbox[3], dx);
        int yi = clamp_axis(y, bbox[1], bbox[4], dy);
        int zi = clamp_axis(z, bbox[2], bbox[5], dz);
        /* local extents at dims {1,1,1}: (hi - lo)/(1*h), truncated */
        int lny = (int)((bbox[4] - bbox[1]) / (1 * dy));
        int lnz = (int)((bbox[5] - bbox[2]) / (1 * dz));
        int idx = xi * lny * lnz + yi * lnz + zi;
        if (idx < 0) idx = 0;
        if (idx >= V) idx = V - 1;
        out_voxel[a] = idx;
    }
}

/* BioFVM_basic_agent.cpp:155-176:
 *   c = dt*volume/dV  (dV = dx*dy*dz, BioFVM_parallel.cpp:156)
 *   temp1 = ((0 + S)*rho*)*c
 *   temp2 = fma(c, U, fma(c, S, 1))   (two axpy calls, fused) */
void orc_agent_constants(int n, int S, double dt, double dx, double dy, double dz,
                         const double *volume, const double *secretion, const double *uptake,
                         const double *saturation, double *temp1, double *temp2)
{
    double dV = dx * dy * dz;
    for (int a = 0; a < n; ++a) {
        double c = dt * volume[a] / dV;
        for (int d = 0; d < S; ++d) {
            size_t e = (size_t)a * S + d;
            double t1 = 0.0;
            t1 += secretion[e];
            t1 *= saturation[e];
            t1 *= c;
            temp1[e] = t1;
            double t2 = 1.0;
            t2 = fma(c, secretion[e], t2);
            t2 = fma(c, uptake[e], t2);
            temp2[e] = t2;
        }
    }
}

/* BioFVM_basic_agent.cpp:291-296: rho += temp1; rho /= temp2, agent by agent. */
void orc_cells_step(double *rho, int S, int n, const int *voxel, const double *temp1,
                    const double *temp2, const uint8_t *active)
{
    for (int a = 0; a < n; ++a) {
        if (active && !active[a]) continue;
        size_t base = (size_t)voxel[a] * S;
        for (int d = 0; d < S; ++d) rho[base + d] += temp1[(size_t)a * S + d];
        for (int d = 0; d < S; ++d) rho[base + d] /= temp2[(size_t)a * S + d];
    }
}

void orc_checksum(const double *rho, int64_t V, int S, double *out)
{
    for (int d = 0; d < S; ++d) out[d] = 0.0;
    for (int64_t v = 0; v < V; ++v)
        for (int d = 0; d < S; ++d) out[d] += rho[(size_t)v * S + d];
}

/* ---------------------------------------------------------------------------
 * Reverse mode of one LOD step (not in the reference; derived from the step
 * above). Per substrate and axis the sweep solves A y = x with the symmetric
 * tridiagonal A = tridiag(-c1, diag, -c1), diag = 1 + 2 c1 + c2 inside and
 * 1 + c1 + c2 at both ends (1 + c2 when n == 1). Dirichlet is the affine
 * overwrite s = (1 - M) y + M g. With lam = dL/ds:
 *   mu = A^{-1} ((1 - M) lam)        (A symmetric, so A^-T = A^-1)
 *   dL/dx = mu,  dL/dc1 -= mu^T Lap y,  dL/dc2 -= mu^T y
 * where Lap = dA/dc1 is tridiag(-1, 2, -1) with end diagonals 1 (0 if n == 1),
 * and c1 = dt D/dx^2, c2 = dt lambda/3.
 * ------------------------------------------------------------------------- */
static int is_active(const uint8_t *face_mask, int S, int d, int i, int j, int k, int nx, int ny, int nz)
{
    for (int f = 0; f < 6; ++f)
        if (face_mask[f * S + d] && on_face(f, i, j, k, nx, ny, nz)) return 1;
    return 0;
}

static void mask_adjoint(double *lam, int nx, int ny, int nz, int S, const uint8_t *face_mask)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < S; ++d)
                    if (is_active(face_mask, S, d, i, j, k, nx, ny, nz))
                        lam[(((size_t)i * ny + j) * nz + k) * S + d] = 0.0;
}

/* Solve in place along every line of one axis with the given factors. */
static void sweep_axis(double *u, int axis, int nx, int ny, int nz, int S,
                       const double *den, const double *c, const double *c1)
{
    size_t ij = (size_t)ny * nz * S, jj = (size_t)nz * S, kj = (size_t)S;
    if (axis == 0) {
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < S; ++d) thomas_line(u, j * jj + k * kj + d, ij, nx, S, d, den, c, c1[d]);
    } else if (axis == 1) {
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < S; ++d) thomas_line(u, i * ij + k * kj + d, jj, ny, S, d, den, c, c1[d]);
    } else {
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int d = 0; d < S; ++d) thomas_line(u, i * ij + j * jj + d, kj, nz, S, d, den, c, c1[d]);
    }
}

/* gD[d] -= (dt/dx^2) mu^T Lap y ; gL[d] -= (dt/3) mu^T y, along one axis. */
static void accumulate_param_grads(const double *mu, const double *y, int axis, int nx, int ny,
                                   int nz, int S, double dt, double dx, double *gD, double *gL)
{
    int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
    size_t stride = axis == 0 ? (size_t)ny * nz * S : (axis == 1 ? (size_t)nz * S : (size_t)S);
    double kD = dt / (dx * dx), kL = dt / 3.0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int m = axis == 0 ? i : (axis == 1 ? j : k);
                size_t vb = (((size_t)i * ny + j) * nz + k) * S;
                for (int d = 0; d < S; ++d) {
                    size_t e = vb + d;
                    double lap = 0.0;
                    if (n > 1) {
                        if (m == 0) lap = y[e] - y[e + stride];
                        else if (m == n - 1) lap = y[e] - y[e - stride];
                        else lap = 2.0 * y[e] - y[e - stride] - y[e + stride];
                    }
                    gD[d] -= kD * mu[e] * lap;
                    gL[d] -= kL * mu[e] * y[e];
                }
            }
}

void orc_lod_step_adjoint(const double *rho_in, double *lam, int nx, int ny, int nz, int S,
                          double dt, double dx, const double *D, const double *lambda,
                          const double *dir_values, const uint8_t *face_mask,
                          double *gD, double *gL)
{
    size_t N = (size_t)nx * ny * nz * S;
    int ns[3] = {nx, ny, nz};
    double *den[3], *cc[3];
    double *c1 = (double *)malloc(sizeof(double) * S);
    orc_constant1(S, dt, dx, D, c1);
    for (int a = 0; a < 3; ++a) {
        den[a] = (double *)malloc(sizeof(double) * ns[a] * S);
        cc[a] = (double *)malloc(sizeof(double) * ns[a] * S);
        orc_factors(ns[a], S, dt, dx, D, lambda, den[a], cc[a]);
    }
    /* replay: y[a] = un-masked solve output of sweep a */
    double *y[3];
    double *s = (double *)malloc(sizeof(double) * N);
    memcpy(s, rho_in, sizeof(double) * N);
    orc_dirichlet(s, nx, ny, nz, S, dir_values, face_mask);
    for (int a = 0; a < 3; ++a) {
        y[a] = (double *)malloc(sizeof(double) * N);
        memcpy(y[a], s, sizeof(double) * N);
        sweep_axis(y[a], a, nx, ny, nz, S, den[a], cc[a], c1);
        memcpy(s, y[a], sizeof(double) * N);
        orc_dirichlet(s, nx, ny, nz, S, dir_values, face_mask);
    }
    for (int a = 2; a >= 0; --a) {
        mask_adjoint(lam, nx, ny, nz, S, face_mask);
        sweep_axis(lam, a, nx, ny, nz, S, den[a], cc[a], c1);
        accumulate_param_grads(lam, y[a], a, nx, ny, nz, S, dt, dx, gD, gL);
    }
    mask_adjoint(lam, nx, ny, nz, S, face_mask);
    for (int a = 0; a < 3; ++a) { free(den[a]); free(cc[a]); free(y[a]); }
    free(s);
    free(c1);
}

/* Microenvironment::compute_all_gradient_vectors (BioFVM_microenvironment.cpp:
 * 1243-1402): per voxel and substrate, out[(n*S + q)*3 + c] =
 *   (rho[+1] - rho[-1]) / (2*h)   inside the axis,
 *   (rho[+1] - rho[ 0]) / h       at the low end,
 *   (rho[ 0] - rho[-1]) / h       at the high end,
 * with h = dx on every axis (uniform mesh; the reference's two_dx is the
 * first call's mesh.dx doubled, :1245-1255), neighbours along x / y / z at
 * ny*nz*S / nz*S / S elements (thomas_i/j/k_jump, BioFVM_parallel.cpp:724-726),
 * each value formed as `g = rho[a]; g -= rho[b]; g /= h` (no contraction).
 * An axis of one voxel has no neighbour: the reference leaves z untouched
 * there (:1352-1354) and reads out of range for x or y; the oracle writes 0
 * for every such axis. */
void orc_gradients(const double *rho, int nx, int ny, int nz, int S, double dx, double *out)
{
    const int ns[3] = {nx, ny, nz};
    const size_t jump[3] = {(size_t)ny * nz * S, (size_t)nz * S, (size_t)S};
    const double two_dx = dx * 2.0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                const int pos[3] = {i, j, k};
                const size_t n = ((size_t)i * ny + j) * nz + k;
                for (int q = 0; q < S; ++q) {
                    const size_t e = n * S + q;
                    for (int c = 0; c < 3; ++c) {
                        double g = 0.0;
                        if (ns[c] > 1) {
                            if (pos[c] == 0) {
                                g = rho[e + jump[c]];
                                g -= rho[e];
                                g /= dx;
                            } else if (pos[c] == ns[c] - 1) {
                                g = rho[e];
                                g -= rho[e - jump[c]];
                                g /= dx;
                            } else {
                                g = rho[e + jump[c]];
                                g -= rho[e - jump[c]];
                                g /= two_dx;
                            }
                        }
                        out[e * 3 + c] = g;
                    }
                }
            }
}

/* ---------------------------------------------------------------------------
 * The product's FP32 path (orc_lod_steps_f32). Not a reference function: the
 * reference has no FP32 solver. Restated from the CUDA line solver so that its
 * results can be checked bit for bit and its error against FP64 predicted on
 * the CPU. Every operation is a single IEEE binary32 operation: the file is
 * compiled with -ffp-contract=off and fused steps call fmaf.
 * ------------------------------------------------------------------------- */

/* The tables of one axis as the host rounds them for the FP32 kernels:
 * rh = RN32(r), rl = RN32(r - rh) with r = 1/den in FP64, a = RN32(c1/den),
 * cb = RN32(c). */
static void f32_tables(int n, int S, const double *den, const double *c, const double *c1, float *rh, float *rl,
                       float *a, float *cb)
{
    for (int m = 0; m < n; ++m)
        for (int d = 0; d < S; ++d) {
            size_t q = (size_t)m * S + d;
            double r = 1.0 / den[q];
            rh[q] = (float)r;
            rl[q] = (float)(r - (double)rh[q]);
            a[q] = (float)(c1[d] / den[q]);
            cb[q] = (float)c[q];
        }
}

/* One line in the deviation form, xb = the line's row 1 (row 0 when n == 1):
 *   p_0 = fma(d_0, rh_0, d_0*rl_0),  p_m = fma(a_m, p_(m-1), fma(d_m, rh_m, d_m*rl_m)),  d_m = x_m - xb
 *   z_(n-1) = p_(n-1),  z_m = fma(-cb_m, z_(m+1), p_m)
 *   out_m = fma(xb, gh, fma(xb, gl, z_m))        (xb*g + z with g = 1/(1+c2) as hi + lo) */
static void thomas_line_f32(float *u, size_t start, size_t stride, int n, int S, int d, const float *rh,
                            const float *rl, const float *a, const float *cb, float gh, float gl, float *p)
{
    const float xb = u[start + (size_t)(n > 1 ? 1 : 0) * stride];
    for (int m = 0; m < n; ++m) {
        const size_t q = (size_t)m * S + d;
        const float dl = u[start + (size_t)m * stride] - xb;
        const float w = fmaf(dl, rh[q], dl * rl[q]);
        p[m] = m == 0 ? w : fmaf(a[q], p[m - 1], w);
    }
    float next = p[n - 1];
    u[start + (size_t)(n - 1) * stride] = fmaf(xb, gh, fmaf(xb, gl, next));
    for (int m = n - 2; m >= 0; --m) {
        next = fmaf(-cb[(size_t)m * S + d], next, p[m]);
        u[start + (size_t)m * stride] = fmaf(xb, gh, fmaf(xb, gl, next));
    }
}

static void dirichlet_f32(float *rho, int nx, int ny, int nz, int S, const float *values, const uint8_t *face_mask)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int face = i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1;
                if (!face) continue;
                size_t base = (((size_t)i * ny + j) * nz + k) * S;
                for (int d = 0; d < S; ++d) {
                    int act = 0;
                    for (int f = 0; f < 6 && !act; ++f)
                        act = face_mask[f * S + d] && on_face(f, i, j, k, nx, ny, nz);
                    if (act) rho[base + d] = values[base + d];
                }
            }
}

void orc_lod_steps_f32(float *rho, int nx, int ny, int nz, int S, double dt, double dx, const double *D,
                       const double *lambda, int n_steps, const double *dir_values, const uint8_t *face_mask)
{
    const int ns[3] = {nx, ny, nz};
    const size_t V = (size_t)nx * ny * nz;
    int nmax = nx > ny ? nx : ny;
    if (nz > nmax) nmax = nz;
    double *den = malloc(sizeof(double) * (size_t)nmax * S), *c = malloc(sizeof(double) * (size_t)nmax * S);
    double *c1 = malloc(sizeof(double) * S);
    float *tab[3][4];
    float *gh = malloc(sizeof(float) * S), *gl = malloc(sizeof(float) * S), *p = malloc(sizeof(float) * nmax);
    float *vals = NULL;
    orc_constant1(S, dt, dx, D, c1);
    for (int ax = 0; ax < 3; ++ax) {
        for (int t = 0; t < 4; ++t) tab[ax][t] = malloc(sizeof(float) * (size_t)ns[ax] * S);
        orc_factors(ns[ax], S, dt, dx, D, lambda, den, c);
        f32_tables(ns[ax], S, den, c, c1, tab[ax][0], tab[ax][1], tab[ax][2], tab[ax][3]);
    }
    for (int d = 0; d < S; ++d) {  /* g = 1/(1 + c2), c2 = dt*lambda/3, as hi + lo */
        double c2 = lambda[d] * dt;
        c2 /= 3.0;
        const double g = 1.0 / (1.0 + c2);
        gh[d] = (float)g;
        gl[d] = (float)(g - (double)gh[d]);
    }
    if (dir_values && face_mask) {
        vals = malloc(sizeof(float) * V * S);
        for (size_t q = 0; q < V * S; ++q) vals[q] = (float)dir_values[q];
    }
    const size_t ij = (size_t)ny * nz * S, jj = (size_t)nz * S, kj = (size_t)S;
    for (int step = 0; step < n_steps; ++step) {
        if (vals) dirichlet_f32(rho, nx, ny, nz, S, vals, face_mask);
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < S; ++d)
                    thomas_line_f32(rho, j * jj + k * kj + d, ij, nx, S, d, tab[0][0], tab[0][1], tab[0][2],
                                    tab[0][3], gh[d], gl[d], p);
        if (vals) dirichlet_f32(rho, nx, ny, nz, S, vals, face_mask);
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < S; ++d)
                    thomas_line_f32(rho, i * ij + k * kj + d, jj, ny, S, d, tab[1][0], tab[1][1], tab[1][2],
                                    tab[1][3], gh[d], gl[d], p);
        if (vals) dirichlet_f32(rho, nx, ny, nz, S, vals, face_mask);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int d = 0; d < S; ++d)
                    thomas_line_f32(rho, i * ij + j * jj + d, kj, nz, S, d, tab[2][0], tab[2][1], tab[2][2],
                                    tab[2][3], gh[d], gl[d], p);
        if (vals) dirichlet_f32(rho, nx, ny, nz, S, vals, face_mask);
    }
    for (int ax = 0; ax < 3; ++ax)
        for (int t = 0; t < 4; ++t) free(tab[ax][t]);
    free(den);
    free(c);
    free(c1);
    free(gh);
    free(gl);
    free(p);
    free(vals);
}

/* The FP32 path's bulk update (not a reference function; the reference's
 * arithmetic is orc_bulk_step's): with A = RN32(T*S) and B = RN32(U + S)
 * formed in FP64 and rounded once, as the host tabulates them, and
 * dt32 = RN32(dt):  rho = RN32(fma(dt32, A, rho) / fma(B, dt32, 1)). */
void orc_bulk_step_f32(float *rho, int64_t V, int S, double dt, const double *S_rate, const double *T_target,
                       const double *U_rate)
{
    const float dt32 = (float)dt;
    for (int64_t e = 0; e < V * S; ++e) {
        const float A = (float)(T_target[e] * S_rate[e]);
        const float B = (float)(U_rate[e] + S_rate[e]);
        rho[e] = fmaf(dt32, A, rho[e]) / fmaf(B, dt32, 1.0f);
    }
}

/* The FP32 path's agent update: simulate_secretion_and_uptake
 * (BioFVM_basic_agent.cpp:291-296) in FP32 for every active agent in list
 * order, rho = (rho + RN32(temp1)) / RN32(temp2), with temp1/temp2 the FP64
 * constants of orc_agent_constants rounded once. */
void orc_cells_step_f32(float *rho, int S, int n, const int *voxel, const double *temp1, const double *temp2,
                        const uint8_t *active)
{
    for (int a = 0; a < n; ++a) {
        if (active && !active[a]) continue;
        for (int d = 0; d < S; ++d) {
            const size_t e = (size_t)voxel[a] * S + d;
            rho[e] = (rho[e] + (float)temp1[(size_t)a * S + d]) / (float)temp2[(size_t)a * S + d];
        }
    }
}

