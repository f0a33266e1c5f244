// Internal declarations shared by the library's translation units.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "minipic_cuda.h"

namespace mp {

// Physical constants exactly as the reference declares them (src/FESolver.h:18-21).
constexpr double EPS0 = 8.8541878e-12;
constexpr double QE = 1.602e-19;
constexpr double AMU = 1.660538921e-27;
constexpr double KB = 8.617333262e-5;

// Device record of one tet for the FP64 walk: the reference's precomputed
// barycentric coefficients (src/meshes.h:38-42), the tet's E field and its
// connectivity, packed so one particle's walk step touches 1.5 cache lines.
struct alignas(64) TetRec {
    double alpha[4];   //   0
    double beta[4];    //  32
    double gamma[4];   //  64
    double delta[4];   //  96
    double ef[3];      // 128
    double volume;     // 152
    int cell_con[4];   // 160
    int con[4];        // 176
};
static_assert(sizeof(TetRec) == 192, "TetRec layout");

// Device record of one tet for the mixed form: FP32 gradients of the four
// barycentric weights (lambda_i = [i==0] + g_i . (x - x_0)), FP32 E field,
// connectivity.  96 B.
struct alignas(32) TetRec32 {
    float gx[4];       //  0  d(lambda_i)/dx
    float gy[4];       // 16
    float gz[4];       // 32
    float ef[3];       // 48
    float pad;         // 60
    int cell_con[4];   // 64
    int con[4];        // 80
};
static_assert(sizeof(TetRec32) == 96, "TetRec32 layout");

// Particle storage, structure of arrays.
struct PartsF64 {
    double *px, *py, *pz, *vx, *vy, *vz;
    int *cell;
    long long *id;
};
struct PartsF32 {
    float *rx, *ry, *rz, *vx, *vy, *vz;   // offsets from the tet's vertex 0, velocities
    int *cell;
    long long *id;
};

// Device counters (one 64-bit word each).
enum Counter {
    C_N = 0,          // particle slots in use (live + holes)
    C_DEAD = 1,       // holes: slots of particles that left the domain
    C_EXITS = 2,      // particles that left this push          } zeroed
    C_HOPS = 3,       // total hops this push                   } before
    C_MAX_HOPS = 4,   // longest walk this push                 } every
    C_NEAR = 5,       // mixed form: FP64 near-face re-tests    } push
    C_FLAGS = 6,      // error bits (FLAG_*), cleared when reported
    C_NEXT_ID = 7,    // next particle id
    C_LOST = 8,       // walks that hit the hop limit and were absorbed (zeroed before every push)
    C_COUNT = 16
};
enum Flag : unsigned long long {
    FLAG_WALK_LIMIT = 1ull,
    FLAG_LOOKBACK_TIMEOUT = 2ull,
    FLAG_SINGULAR = 4ull,
    FLAG_NONFINITE = 8ull,
    FLAG_BAD_INDEX = 16ull,   // a cell, neighbour or node index outside the mesh (caller-owned records)
    FLAG_HALF_RANGE = 32ull,  // an FP16 operand of the mixed factorization's update would overflow
};

// The per-quadrature-point shape function values used by buildF1Vector and
// buildJmatrix (src/FESolver.cpp:497-501, 604-609): Na[a][p], p in the
// reference's k,j,i loop order.
struct Quadrature {
    double Na[4][8];
};
Quadrature make_quadrature();

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
};

// Device time of kernel classes (mp_set_kernel_timing): launches, summed CUDA
// event time, summed algorithmic work (bytes for the push, flops for the
// trailing updates).
struct KernelClock {
    long long launches = 0;
    double ms = 0, work = 0;
};
struct KernelMark {
    int cls;
    double work;
    cudaEvent_t a, b;
};

}  // namespace mp

struct mp_ctx {
    int device = 0;
    int sm_count = 0;
    int push_grid[2] = {0, 0};
    cudaStream_t stream = nullptr;
    std::string last_error;

    // mesh
    int n_nodes = 0, n_tets = 0;
    bool small_tets = false;              // every tet volume < 1: exact division-free inside test
    mp::TetRec *tets = nullptr;           // [n_tets]
    mp::TetRec32 *tets32 = nullptr;       // [n_tets] (mixed form)
    double *tet_x0 = nullptr;             // [n_tets][4] vertex 0 position (x,y,z,pad)
    double *node_volume = nullptr;        // [n_nodes]
    double *node_pos = nullptr;           // [n_nodes][3]
    double *ef = nullptr;                 // [n_tets][3]
    int *con = nullptr;                   // [n_tets][4]
    double *den = nullptr;                // [n_nodes]
    double *den_in = nullptr;             // [n_nodes] host-supplied density for computePhi
    unsigned long long *den_fixed = nullptr;  // [n_nodes] fixed-point accumulator

    // particles
    int form = MP_FORM_FP64;
    int scatter_mode = MP_SCATTER_FP64_ATOMIC;
    int walk_limit = 4096;
    bool walk_absorb = false;             // hop limit: absorb the particle instead of raising MP_ERR_WALK_LIMIT
    int sort_period = 0;
    int mixed_factor = MP_MIXED_AUTO;    // tensor-core terms of the mixed factorization
    long long steps_since_sort = 0;
    bool track_ids = true;
    long long capacity = 0;
    long long n_host = 0;                 // particle slots (live + holes); exact after a sync, else an upper bound
    long long dead_host = 0;              // holes, as of the last sync
    int *compact_off = nullptr;           // per-block offsets of the stable compaction
    long long compact_len = 0;
    mp::PartsF64 p64[2] = {};
    mp::PartsF32 p32[2] = {};
    int cur = 0;                          // which buffer holds the live particles
    void *part_block[2] = {nullptr, nullptr};
    unsigned long long *counters = nullptr;     // device [C_COUNT]
    unsigned long long *counters_host = nullptr;  // pinned mirror
    // pinned staging for host appends/downloads
    void *stage = nullptr;
    size_t stage_bytes = 0;
    // sort scratch
    int *sort_hist = nullptr;
    void *sort_tmp = nullptr;

    // FE
    bool fe_ready = false;
    int neq = 0;
    double n0 = 0, phi0 = 0, kTe = 0;
    int *ID = nullptr;            // [n_nodes]
    int *LM = nullptr;            // [n_tets][4]
    double *detJ = nullptr;       // [n_tets]
    double *nx = nullptr;         // [n_tets][12]
    double *g = nullptr, *uh = nullptr;   // [n_nodes]
    double *d = nullptr, *F0 = nullptr, *F1 = nullptr, *G = nullptr, *y = nullptr;  // [neq]
    double *fvec = nullptr, *FP = nullptr, *work = nullptr;  // [neq]
    double *K = nullptr, *J = nullptr;    // [neq][neq] row-major
    float *J32 = nullptr;                 // [neq][neq] mixed-form factor
    float *K32 = nullptr;                 // [neq][neq] K's lower triangle in FP32 (the mixed form's J32 source)
    bool k32_current = false;             // K32 holds the current K
    bool j32_current = false;             // J32 holds the lower triangle of the current J
    bool j_current = false;               // J holds the current J (not yet overwritten by its factor)
    double *scal = nullptr;               // device scalars for reductions
    double *scal_host = nullptr;          // pinned
    int *eq_ptr = nullptr, *eq_tet = nullptr;   // CSR equation -> (tet, a) sorted by tet
    unsigned char *eq_a = nullptr;
    double *gs_minv = nullptr;            // Gauss-Seidel: (D+L)^-1, [neq][neq]
    // sparse K, sliced ELLPACK (slices of 32 rows): entry k of row P (columns
    // ascending) at sp_ptr[P >> 5] + 32 * k + (P & 31); padding col = P, val = 0
    int fe_storage = MP_FE_STORAGE_DENSE;
    int *sp_len = nullptr;                // [neq] nonzeros of each row
    long long *sp_ptr = nullptr;          // [slices + 1]
    int *sp_col = nullptr;                // [sp_slots]
    double *sp_val = nullptr;             // [sp_slots]
    long long sp_nnz = 0, sp_slots = 0;
    void *sparse_scratch = nullptr;       // conjugate-gradient work (mp_sparse.cu)
    double cg_rtol = 1e-12;               // ||G - J y|| <= cg_rtol ||G||
    int cg_max_it = 20000;
    int gs_max_sweeps = 10000;            // solveLinear's sweep limit (src/FESolver.cpp:575)
    int cg_last_iterations = 0, cg_last_restarts = 0;
    double cg_last_relres = 0;

    // dense-solve scratch (mp_solve.cu): W panels, block inverses, ready words;
    // sized for neq, allocated on the first factorization
    void *solve_scratch = nullptr;
    int solve_epoch = 0;                  // epoch of this context's wavefront words (solves, sweeps)
    bool ldlt_attr = false;               // >48 KB shared-memory attributes set for this context's device
    // device staging of host appends and downloads
    void *dstage = nullptr;
    size_t dstage_bytes = 0;

    mp::Timer t0, t1, tp, ts;
    long long launches = 0;
    // kernel-class timing, off unless asked for (mp_set_kernel_timing)
    unsigned ktime_mask = 0;              // bit k: kernel class k timed
    mp::KernelClock kclock[8];
    std::vector<mp::KernelMark> kmarks;     // recorded, not yet read
    std::vector<cudaEvent_t> kevents;       // free events

    void *adjoint = nullptr;              // adjoint state (mp_adjoint.cu), created by mp_adjoint_setup
    void *inject = nullptr;               // device injection state (mp_inject.cu)
    void *output = nullptr;               // VTK output state and writer thread (mp_output.cpp)
};

namespace mp {

int fail(mp_ctx *ctx, int code, const std::string &msg);

// Kernel-class timing: kt_begin records an event before a launch (returns a
// mark index, or -1 when timing is off), kt_end one after it; kt_collect reads
// the marks whose events have completed (call after a stream synchronise).
int kt_begin(mp_ctx *ctx, int cls, double work);
void kt_end(mp_ctx *ctx, int mark);
void kt_collect(mp_ctx *ctx);
int cuda_fail(mp_ctx *ctx, cudaError_t e, const char *what);

#define MP_CUDA(ctx, call)                                  \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return mp::cuda_fail((ctx), e_, #call); \
    } while (0)

// Kernels' host launchers (push / field / solver translation units).
int launch_push(mp_ctx *ctx, double q_over_m, double dt);
int launch_normalise(mp_ctx *ctx, double spwt);
int launch_append(mp_ctx *ctx, long long n, const double *pos_soa, const double *vel_soa, const int *cell,
                  int rewind, double q_over_m, double half_dt);
int launch_download_pack(mp_ctx *ctx, long long n, double *out_soa /*3+3+4 arrays*/, int *cell_out,
                         long long *id_out);
int launch_sort_by_tet(mp_ctx *ctx);
int launch_compact(mp_ctx *ctx);
int launch_convert_form(mp_ctx *ctx, int to_form);
int launch_update_ef(mp_ctx *ctx);

int fe_build_f1(mp_ctx *ctx, const double *den_dev);
int fe_residual(mp_ctx *ctx);
int fe_build_j(mp_ctx *ctx, int method, int form = MP_FORM_FP64);
int fe_j32_from_k(mp_ctx *ctx);
int fe_solve_ldlt(mp_ctx *ctx, int form, mp_newton_stats *st);
int fe_solve_gs(mp_ctx *ctx, mp_newton_stats *st);
int fe_update_d(mp_ctx *ctx, double *l2_out);
int fe_uh(mp_ctx *ctx);
int fe_assemble(mp_ctx *ctx);
int sparse_setup(mp_ctx *ctx, const std::vector<int> &LM, const std::vector<int> &eq_ptr,
                 const std::vector<int> &eq_tet);
void sparse_free(mp_ctx *ctx);
int fe_assemble_sparse(mp_ctx *ctx);
int fe_sparse_from_dense(mp_ctx *ctx);
int fe_sparse_from_host(mp_ctx *ctx, const double *const *rows, const double *dense);
int fe_residual_sparse(mp_ctx *ctx);
int fe_resid_j_sparse(mp_ctx *ctx, const double *y, const double *b, double *r, float *r32, double *sums);
int fe_solve_cg(mp_ctx *ctx, mp_newton_stats *st);
void solve_free(mp_ctx *ctx);
void adjoint_free(mp_ctx *ctx);
void inject_free(mp_ctx *ctx);
void output_free(mp_ctx *ctx);

}  // namespace mp
