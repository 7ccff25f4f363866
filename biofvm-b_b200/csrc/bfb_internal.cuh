// bfb_internal.cuh -- shared types of the B200 diffusion-decay library.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "biofvm_b200.h"

namespace bfb {

// An NVTX range over a host scope: one per entry point that launches work and
// one per phase in bfb_profile_steps, so that profilers recording NVTX (ncu's
// --nvtx filters) can select them. Without a profiler attached the calls do
// nothing.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// ---------------------------------------------------------------------------
// Error plumbing: every C entry point returns a status and records a message.
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

// Waits for the env's stream, then reads its sticky device error flag:
// BFB_ERR_WATCHDOG once a kernel's bounded wait has run out (the field is then
// not trustworthy), BFB_OK otherwise.
int env_check_device_error(::bfb_env_s *env);

#define BFB_CUDA(call)                                        \
    do {                                                      \
        cudaError_t _e = (call);                              \
        if (_e != cudaSuccess) return ::bfb::cuda_fail(_e, #call); \
    } while (0)

// ---------------------------------------------------------------------------
// Dirichlet faces on the device.
//   faces[f] holds the values of face f for every substrate:
//     f = 0/1 (x-lo/hi): [ny][nz][S]   f = 2/3 (y-lo/hi): [nx][nz][S]
//     f = 4/5 (z-lo/hi): [nx][ny][S]
//   mask[d] bit f set <=> face f is active for substrate d.
// A voxel on several faces (edges, corners) has the same value in every face
// array, because all are cut from one per-voxel array.
// ---------------------------------------------------------------------------
// The field element of voxel v = (i*ny + j)*nz + k, substrate d, with the
// (i, j) rows Lp elements apart.
__device__ __forceinline__ size_t voxel_elem(int v, int d, int nz, int S, int Lp) {
    const int row = v / nz;
    return (size_t)row * Lp + (size_t)(v - row * nz) * S + d;
}

template <typename T>
struct DirFaces {
    const T *face[6];
    const uint8_t *mask;  // [S]
    int nx, ny, nz, S;
    int any;              // 0: no active face for any substrate
};

// Bulk source/sink terms fused into the x-sweep load.
//   A = S*T (rounded once), B = U + S (rounded once); rho <- (rho + dt*A) / (B*dt + 1)
template <typename T>
struct BulkTerms {
    const T *A;
    const T *B;
    T dt;
    int on;
};

// Launch shape of the three sweeps, chosen by bfb_autotune or set by
// bfb_set_tuning. Every shape computes the same numbers; only speed differs.
struct SweepTuning {
    int tma[3] = {1, 1, 1};     // TMA tiles (when the grid allows them) or cp.async tiles
    int warps[3] = {1, 1, 1};   // warps (= tiles) per CTA; one packs shared memory tightest
    int chunks[3] = {2, 2, 2};  // row groups per TMA tile (pipeline stages); 2 measured fastest
};

}  // namespace bfb

// ---------------------------------------------------------------------------
// The environment handle.
// ---------------------------------------------------------------------------
struct bfb_env_s {
    int device = 0;
    int precision = BFB_FP64;
    int nx = 0, ny = 0, nz = 0, S = 0;
    double dx = 0;
    double bbox[6] = {0, 0, 0, 0, 0, 0};  // x0, y0, z0, x1, y1, z1
    cudaStream_t stream = nullptr;       // stream all device work is issued on
    cudaStream_t own_stream = nullptr;   // created by bfb_create, used unless bfb_set_stream overrides
    size_t elem = 8;                     // bytes per field element
    int64_t V = 0;                       // voxels
    int64_t N = 0;                       // V * S (the packed, reference layout)
    // Row pitch of the device field: the nz*S values of an (i, j) row are
    // followed by padding up to a whole number of 16-byte vectors when nz*S*elem
    // is not one (so that every sweep can use the TMA tiles); Lp = nz*S
    // otherwise. rho(i,j,k,d) lives at (i*ny + j)*Lp + k*S + d, and the field
    // holds Np = nx*ny*Lp elements.
    int Lp = 0;
    int64_t Np = 0;

    void *field = nullptr;               // device, N elements
    void *staging = nullptr;             // device, N doubles (host double <-> env precision)

    // coefficients and cached factors
    std::vector<double> D, lambda;
    bool factors_valid = false;
    double factor_dt = 0;
    int freeze_factors = 1;
    // per axis: tables [4][n*S] (FP64 uses 2: den, c; FP32 uses 4: 1/den hi,
    // 1/den lo, c1/den, c) and tail values [4][S] for rows [m0, n-2]
    void *fac_tab[3] = {nullptr, nullptr, nullptr};
    void *fac_tail[3] = {nullptr, nullptr, nullptr};
    void *fac_head[3] = {nullptr, nullptr, nullptr};
    int fac_hpad[3] = {4, 4, 4};
    int fac_m0[3] = {1, 1, 1};
    void *c1 = nullptr;                  // [S] (FP64)
    void *g = nullptr;                   // [2*S] (FP32): 1/(1 + c2) as hi, lo

    // Dirichlet
    std::vector<uint8_t> activation;     // [S]
    std::vector<uint8_t> face_mask;      // [6*S], already ANDed with activation
    void *faces[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    uint8_t *d_mask = nullptr;           // [S]
    int dir_any = 0;

    // bulk
    int bulk_on = 0;
    void *bulkA = nullptr, *bulkB = nullptr;

    // agents
    int n_agents = 0;
    int n_occ = 0;                       // occupied voxels with >= 1 active agent
    int *agent_voxel = nullptr;          // [n_agents], list order (current_voxel_index)
    int *seg_start = nullptr;            // [n_occ + 1]
    int *seg_voxel = nullptr;            // [n_occ]
    void *ag_t1 = nullptr, *ag_t2 = nullptr;  // [n_active][S] in voxel-sorted, list-stable order
    int n_active = 0;
    int *ag_order = nullptr;             // [n_active]: list index of each sorted agent
    // rates as given to bfb_set_agents (list order), for the adjoint's chain rule
    std::vector<double> h_vol, h_sec, h_upt, h_sat;
    double agent_dt = 0;

    // scratch for reductions
    double *partials = nullptr;
    int partial_blocks = 0;

    // CUDA graph of bfb_simulate
    int use_graphs = 1;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_flags = -1;
    double graph_dt = 0;
    uint64_t graph_epoch = 0;            // bumps whenever captured state changes
    uint64_t epoch = 1;

    bfb::SweepTuning tuning;

    // TMA: tensor maps of the field for the x and y sweeps (made at creation
    // when the grid meets TMA's alignment rules), and the switch
    int use_tma = 1;
    CUtensorMap tmap[2];
    int tma_crow[2] = {0, 0};
    int tma_lines[2] = {32, 32};  // lines per warp tile of the maps' boxes
    int tma_ok[2] = {0, 0};
    // FP64: maps of 16-row boxes for the tensor-memory x/y sweeps (tuning tma = 2)
    CUtensorMap tmem_map[2];
    int tmem_ok[2] = {0, 0};

    // sticky device error flag (a bounded wait in a kernel ran out)
    int *d_err = nullptr;

    // x-slab of a larger grid (bfb_create_slab): planes [x0, x0 + nx) of
    // nx_global; 0 for a whole grid
    int nx_global = 0;
    int x0 = 0;

    // reverse-mode workspace (bfb_adjoint.cu): one device block, kept between
    // calls and grown on demand, freed by bfb_destroy
    void *adj_ws = nullptr;
    size_t adj_ws_bytes = 0;
};
