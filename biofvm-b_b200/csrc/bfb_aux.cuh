// bfb_aux.cuh -- agents, reductions and conversions.
#pragma once
#include "bfb_internal.cuh"

namespace bfb {

// Field precision conversion (device).
int launch_convert_d2f(const double *src, float *dst, long long n, cudaStream_t s);
int launch_convert_f2d(const float *src, double *dst, long long n, cudaStream_t s);
// The same over `rows` rows of L elements, src rows `sp` and dst rows `dp`
// elements apart (packed V*S <-> a field with padded rows).
int launch_convert_d2f_rows(const double *src, float *dst, long long rows, int L, int sp, int dp, cudaStream_t s);
int launch_convert_f2d_rows(const float *src, double *dst, long long rows, int L, int sp, int dp, cudaStream_t s);

// Agents: binning + cached constants (FP64, bit-exact with the reference),
// then a stable voxel sort and per-voxel segments. All device memory of the
// previous agent set is released first.
int agents_build(bfb_env_s *env, int n, const double *pos, const double *volume, const double *sec,
                 const double *upt, const double *sat, const uint8_t *active, double dt);
// Same, from the constants an agent already caches (current_voxel_index,
// temp1, temp2 in list order), as the reference's Basic_Agent holds them.
int agents_build_constants(bfb_env_s *env, int n, const int *voxel, const double *t1, const double *t2,
                           const uint8_t *active);
void agents_free(bfb_env_s *env);
int launch_cells(bfb_env_s *env, cudaStream_t s);

// Per-substrate FP64 sums of the field. Writes S doubles to out_dev. Uses
// env->partials (allocated on demand, outside any stream capture).
int checksum_prepare(bfb_env_s *env);
int launch_checksum(bfb_env_s *env, double *out_dev, cudaStream_t s);
// max|a-b|, max|b|, sum (a-b)^2, sum b^2 of two device fields of `rows` rows
// of L elements, a's rows la and b's rows lb elements apart.
int compare_fields(const void *a, int pa, int la, const void *b, int pb, int lb, long long rows, int L, double *out4,
                   cudaStream_t s);
// The same kernels on caller-provided scratch (partials: nblocks*S doubles).
int launch_checksum_raw(const void *field, int precision, long long V, int S, double *partials, int nblocks,
                        double *out_dev, cudaStream_t s);

}  // namespace bfb
