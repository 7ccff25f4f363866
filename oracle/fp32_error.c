/* fp32_error.c -- the FP32 path's error against FP64 on the CPU, from the
 * oracle's FP64 LOD step (orc_lod_step's line solver) and the FP32 path's
 * restatement (orc_lod_steps_f32's line solver), lines in parallel with
 * OpenMP; each line's arithmetic is that of the oracle, unchanged. No
 * Dirichlet faces. Test infrastructure: built by `make -C oracle fp32err`,
 * fed by fp32_error_input.py.
 *
 *   python oracle/fp32_error_input.py 256 555 /tmp/in.bin && oracle/_build/fp32_error /tmp/in.bin
 *
 * Input: int nx, ny, nz, S, steps; double D[S], lambda[S]; double rho0[V*S]
 * (dt = 0.01, dx = 20). Output: the relative L-inf (max|f32 - f64| / max|f64|,
 * order-independent) and relative L2 of the FP32 field against the FP64 one.
 */
#include "lod_oracle.c"
#include <omp.h>
#include <stdio.h>

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: fp32_error <input.bin>\n");
        return 2;
    }
    FILE *fp = fopen(argv[1], "rb");
    if (!fp) return 2;
    int hdr[5];
    if (fread(hdr, sizeof(int), 5, fp) != 5) return 1;
    int nx = hdr[0], ny = hdr[1], nz = hdr[2], S = hdr[3], steps = hdr[4];
    if (nx < 1 || ny < 1 || nz < 1 || S < 1 || nx > 1024 || ny > 1024 || nz > 1024) {
        fprintf(stderr, "axes of 1..1024 voxels (the per-line scratch holds 1024 rows)\n");
        return 2;
    }
    double *D = malloc(8 * S), *lam = malloc(8 * S);
    if (fread(D, 8, S, fp) != (size_t)S || fread(lam, 8, S, fp) != (size_t)S) return 1;
    size_t V = (size_t)nx * ny * nz, N = V * S;
    double *r64 = malloc(8 * N);
    if (fread(r64, 8, N, fp) != N) return 1;
    fclose(fp);
    float *r32 = malloc(4 * N);
    for (size_t q = 0; q < N; ++q) r32[q] = (float)r64[q];
    const double dt = 0.01, dx = 20.0;
    const int ns[3] = {nx, ny, nz};
    double *den[3], *cc[3], *c1 = malloc(8 * S);
    float *tab[3][4], *gh = malloc(4 * S), *gl = malloc(4 * S);
    orc_constant1(S, dt, dx, D, c1);
    for (int a = 0; a < 3; ++a) {
        den[a] = malloc(8 * (size_t)ns[a] * S);
        cc[a] = malloc(8 * (size_t)ns[a] * S);
        orc_factors(ns[a], S, dt, dx, D, lam, den[a], cc[a]);
        for (int t = 0; t < 4; ++t) tab[a][t] = malloc(4 * (size_t)ns[a] * S);
        f32_tables(ns[a], S, den[a], cc[a], c1, tab[a][0], tab[a][1], tab[a][2], tab[a][3]);
    }
    for (int d = 0; d < S; ++d) {
        double c2 = lam[d] * dt;
        c2 /= 3.0;
        const double g = 1.0 / (1.0 + c2);
        gh[d] = (float)g;
        gl[d] = (float)(g - (double)gh[d]);
    }
    const size_t ij = (size_t)ny * nz * S, jj = (size_t)nz * S, kj = (size_t)S;
    double t0 = omp_get_wtime();
    for (int s = 0; s < steps; ++s) {
        #pragma omp parallel for collapse(2) schedule(static)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < S; ++d) {
                    float p[1024];
                    thomas_line(r64, j * jj + k * kj + d, ij, nx, S, d, den[0], cc[0], c1[d]);
                    thomas_line_f32(r32, j * jj + k * kj + d, ij, nx, S, d, tab[0][0], tab[0][1], tab[0][2], tab[0][3], gh[d], gl[d], p);
                }
        #pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < S; ++d) {
                    float p[1024];
                    thomas_line(r64, i * ij + k * kj + d, jj, ny, S, d, den[1], cc[1], c1[d]);
                    thomas_line_f32(r32, i * ij + k * kj + d, jj, ny, S, d, tab[1][0], tab[1][1], tab[1][2], tab[1][3], gh[d], gl[d], p);
                }
        #pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int d = 0; d < S; ++d) {
                    float p[1024];
                    thomas_line(r64, i * ij + j * jj + d, kj, nz, S, d, den[2], cc[2], c1[d]);
                    thomas_line_f32(r32, i * ij + j * jj + d, kj, nz, S, d, tab[2][0], tab[2][1], tab[2][2], tab[2][3], gh[d], gl[d], p);
                }
        if (s == 0 || (s + 1) % 50 == 0) fprintf(stderr, "step %d %.1f s\n", s + 1, omp_get_wtime() - t0);
    }
    double mx = 0, mb = 0, sd = 0, sb = 0;
    for (size_t q = 0; q < N; ++q) {
        const double x = (double)r32[q], y = r64[q], df = x - y;
        mx = fmax(mx, fabs(df));
        mb = fmax(mb, fabs(y));
        sd += df * df;
        sb += y * y;
    }
    printf("rel_linf %.17g rel_l2 %.17g\n", mx / mb, sqrt(sd / sb));
    return 0;
}
