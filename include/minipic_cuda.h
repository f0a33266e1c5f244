/* minipic_cuda.h -- C ABI of the B200 (sm_100a) implementation of mini-pic's
 * per-step hot path: particle push + barycentric tet walk + node-density
 * scatter (MoveParticles), the per-element E-field gather (FESolver::updateEf)
 * and FESolver's Poisson-Boltzmann Newton step (computePhi).
 *
 * Plain pointers and sizes only.  Every call returns an int status (MP_OK or
 * an MP_ERR_* code); mp_last_error() gives the message of the last failure on
 * a context.  One context per host thread; a context owns one CUDA stream and
 * all of its device buffers.  There is no CPU fallback: without a usable
 * sm_100 device mp_create returns MP_ERR_NO_DEVICE.
 *
 * Reference interfaces each entry point replaces (paths in the reference
 * project AD1641/mini-fem-pic-main):
 *   mp_create / mp_destroy        DeviceData ctor/dtor, src/mini-pic.cpp:322-345
 *   mp_particles_append           InjectIons' push_back + the per-step H2D copy,
 *                                 src/mini-pic.cpp:257-260, 274-275
 *   mp_push_scatter               MoveParticles, src/mini-pic.cpp:268-320
 *   mp_particles_download         the per-step D2H copy, src/mini-pic.cpp:311
 *   mp_density_download           src/mini-pic.cpp:312
 *   mp_fe_setup                   FESolver ctor + preAssembly, src/FESolver.cpp:48-127, 434-485
 *   mp_compute_phi                FESolver::computePhi, src/FESolver.cpp:604-619
 *   mp_fe_build_f1                FESolver::buildF1Vector, src/FESolver.cpp:488-526
 *   mp_fe_residual                G = K d - F0 - F1, src/FESolver.cpp:333-335
 *   mp_fe_build_j                 FESolver::buildJmatrix, src/FESolver.cpp:367-431
 *   mp_fe_solve_linear            FESolver::solveLinear / solveLinearLapack,
 *                                 src/FESolver.cpp:561-601 / 528-558
 *   mp_update_ef                  FESolver::updateEf, src/FESolver.cpp:622-636
 *   mp_field_download             reads of FESolver::d, uh, ef (src/FESolver.h:45-49)
 *   mp_mesh_geometry              LoadVolumeMesh geometry precompute, src/meshes.cpp:87-251
 *   mp_fe_geometry                FESolver::computeNX + ID/LM, src/FESolver.cpp:108-118, 207-287
 *   mp_injector_*                 InjectIons, src/mini-pic.cpp:208-265
 *   mp_adjoint_*                  no reference counterpart: derivatives of K steps of
 *                                 MoveParticles + InjectIons (src/mini-pic.cpp:208-320)
 *                                 with respect to the node potential and the drift
 *   mp_set_fe_storage,            sparse K (preAssembly's K, src/FESolver.cpp:434-485,
 *   mp_fe_sparse_matrix           without its zeros) and the SPARSE_* methods
 *   mp_*_geometry_device,         the three geometry helpers above, on the device
 *   mp_inlet_faces_device
 *   mp_output_mesh                OutputMesh, src/meshes.cpp:358-447 (asynchronous)
 *   mp_output_particles           OutputParticles, src/particles.cpp:21-45
 */
#ifndef MINIPIC_CUDA_H
#define MINIPIC_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
enum {
    MP_OK = 0,
    MP_ERR_ARG = 1,           /* bad argument (null pointer, size, index) */
    MP_ERR_OOM = 2,           /* device or pinned-host allocation failed */
    MP_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    MP_ERR_WALK_LIMIT = 4,    /* a particle's tet walk exceeded the hop limit */
    MP_ERR_NOT_CONVERGED = 5, /* Newton (NonLinear method) did not converge */
    MP_ERR_SINGULAR = 6,      /* factorization met a zero/non-finite pivot */
    MP_ERR_STATE = 7,         /* call out of order (e.g. no FE setup yet) */
    MP_ERR_NO_DEVICE = 8,     /* no usable sm_100 device */
    MP_ERR_TIMEOUT = 9,       /* a bounded device-side wait gave up */
    MP_ERR_LIMIT = 10         /* size above the fixed maximum of an allocation-free entry point */
};

/* FESolver::Method, src/FESolver.h:26, and two sparse methods of this library:
 * SPARSE_CG is the Lapack method's single Newton step (src/FESolver.cpp:301-317)
 * with J y = G solved by Jacobi-preconditioned conjugate gradients in FP64 on
 * the sparse K (||G - J y|| <= rtol ||G||, mp_set_sparse_solver);
 * SPARSE_NEWTON is the NonLinear method's loop (src/FESolver.cpp:324-364: F1
 * accumulating, up to 10 iterations, stop at ||y||/neq < 1e-2) with the same
 * conjugate-gradient inner solves in place of Gauss-Seidel. */
enum {
    MP_METHOD_NONLINEAR = 0, MP_METHOD_GAUSS_SEIDEL = 1, MP_METHOD_LAPACK = 2,
    MP_METHOD_SPARSE_CG = 3, MP_METHOD_SPARSE_NEWTON = 4
};

/* Storage of K for the field solve.  DENSE (the reference's neq x neq arrays,
 * src/FESolver.cpp:80-127) keeps a sparse copy beside it, so every method
 * runs; SPARSE keeps only the sparse K (about 15 nonzeros a row, 12 B each)
 * and runs the SPARSE_* methods, for meshes whose dense K does not fit. */
enum { MP_FE_STORAGE_DENSE = 0, MP_FE_STORAGE_SPARSE = 1 };

/* Arithmetic forms. FP64 is the reference's method bit for bit on the particle
 * side; MIXED stores particles as FP32 offsets from the owning tet's vertex 0
 * (FP64 near-face re-test, FP64 density accumulators) and factors the Newton
 * Jacobian in TF32 on the tensor cores with FP64 iterative refinement. */
enum { MP_FORM_FP64 = 0, MP_FORM_MIXED = 1 };

/* Tensor-core arithmetic of the mixed form's FP32 factorization: one TF32
 * product per term, or the 3xTF32 split (hi*hi + hi*lo + lo*hi, about FP32
 * accuracy; fewer FP64 refinement iterations). */
enum { MP_MIXED_AUTO = 0, MP_MIXED_TF32 = 1, MP_MIXED_FP16 = 2, MP_MIXED_TF32X3 = 3 };

/* What a walk that reaches the hop limit does.  In a mesh with a cavity (the
 * sphere workload) a particle that steps into the cavity lies in no tet, and
 * the reference's greedy XtoLtet walk (src/meshes.h:75-100) can then cycle
 * among the tets around it without end.  ERROR keeps the particle where the
 * walk stopped and returns MP_ERR_WALK_LIMIT; ABSORB removes it as absorbed by
 * the boundary and counts it in mp_step_stats.lost. */
enum { MP_WALK_LIMIT_ERROR = 0, MP_WALK_LIMIT_ABSORB = 1 };

/* Density accumulation: FP64 atomics (order-dependent rounding, like the
 * reference's atomic_ref) or 64-bit fixed point (run-to-run deterministic). */
enum { MP_SCATTER_FP64_ATOMIC = 0, MP_SCATTER_FIXED64 = 1 };

/* Particle order for mp_particles_download. */
enum { MP_ORDER_STORAGE = 0, MP_ORDER_ID = 1 };

/* Vector/matrix names for mp_fe_download / mp_fe_upload. */
enum {
    MP_VEC_F0 = 0, MP_VEC_F1 = 1, MP_VEC_D = 2, MP_VEC_G = 3, MP_VEC_UH = 4,
    MP_VEC_DEN = 5, MP_VEC_EF = 6, MP_VEC_RESIDUAL = 7, MP_VEC_Y = 8,
    MP_MAT_K = 16, MP_MAT_J = 17
};

typedef struct mp_ctx mp_ctx;

/* Mesh description.  Every per-tet field is given by the address of tet 0's
 * field and the byte stride between consecutive tets, so a caller can point
 * straight into an array of the reference's Tetra records (stride 168) or
 * into packed arrays.  Same for per-node fields (the reference's Node is 40 B). */
typedef struct mp_mesh_desc {
    int32_t n_nodes;
    int32_t n_tets;
    const int32_t *con;      int64_t con_stride;      /* 4 node ids, src/meshes.h:34 */
    const double *volume;    int64_t volume_stride;   /* src/meshes.h:35 */
    const double *alpha;     int64_t alpha_stride;    /* 4 each, src/meshes.h:39 */
    const double *beta;      int64_t beta_stride;
    const double *gamma;     int64_t gamma_stride;
    const double *delta;     int64_t delta_stride;
    const int32_t *cell_con; int64_t cell_con_stride; /* 4 neighbours, -1 = none, src/meshes.h:42 */
    const double *node_pos;  int64_t node_pos_stride; /* 3 coords, src/meshes.h:27 */
    const double *node_volume; int64_t node_volume_stride; /* src/meshes.h:29 */
} mp_mesh_desc;

/* FE description (FESolver's public members, src/FESolver.h:27-51). */
typedef struct mp_fe_desc {
    int32_t neq;
    const int32_t *ID;        /* [n_nodes] equation of each node, -1 = Dirichlet */
    const double *nx;         /* [n_tets][4][3] dN_a/dx (FESolver::NX) */
    const double *detJ;       /* [n_tets] */
    const double *g;          /* [n_nodes] Dirichlet values */
    const double *const *K_rows; /* optional: neq row pointers of K; NULL = assemble on the device */
    const double *K_dense;    /* optional alternative: row-major neq x neq */
    const double *F0;         /* optional [neq]; NULL = assemble on the device */
    double n0, phi0, kTe;     /* Boltzmann reference values */
} mp_fe_desc;

typedef struct mp_step_stats {
    int64_t n_before;         /* particles pushed */
    int64_t n_after;          /* particles kept */
    int64_t total_hops;       /* tet-to-tet moves of all particles this step */
    int32_t max_hops;         /* longest walk this step */
    int32_t near_face_fp64;   /* mixed form: FP64 re-tests taken */
    double ms_kernel;         /* device time of the push kernel alone (CUDA events) */
    double ms_step;           /* device time of the whole push call's kernels */
    int64_t lost;             /* walks that hit the hop limit and were absorbed (MP_WALK_LIMIT_ABSORB) */
} mp_step_stats;

typedef struct mp_newton_stats {
    int32_t newton_iterations;
    int32_t linear_iterations;   /* GS sweeps of the last solve / refinement steps */
    double l2;                   /* ||y|| / neq of the last Newton update */
    double linear_residual;      /* ||b - J y|| / neq of the last linear solve */
    double ms_total;             /* device time of the call, ms */
    double ms_factor;            /* device time of the factorization, ms */
    int32_t linear_failures;     /* Gauss-Seidel solves that ran out of sweeps above the tolerance
                                    (the reference warns "GS failed to converge" and goes on,
                                    src/FESolver.cpp:600) */
    int32_t reserved;
} mp_newton_stats;

/* ---- context ---------------------------------------------------------------- */
const char *mp_error_string(int status);
const char *mp_last_error(const mp_ctx *ctx);
int mp_version(void);

int mp_create(int device, const mp_mesh_desc *mesh, mp_ctx **out);
int mp_destroy(mp_ctx *ctx);
int mp_synchronize(mp_ctx *ctx);
int mp_get_stream(mp_ctx *ctx, void **cuda_stream);
/* Options: hop limit of the tet walk (default 4096), density accumulation mode,
 * particle-ID tracking (default on), tet re-sort period in steps (0 = never). */
int mp_set_walk_limit(mp_ctx *ctx, int32_t max_hops);
int mp_set_scatter_mode(mp_ctx *ctx, int mode);
int mp_set_walk_policy(mp_ctx *ctx, int policy);
int mp_set_sort_period(mp_ctx *ctx, int32_t steps);
/* Particle storage of the push (MoveParticles, src/mini-pic.cpp:268-320):
 * MP_FORM_FP64 (default) is the reference's arithmetic bit for bit; with
 * MP_FORM_MIXED positions are FP32 offsets from the owning tet's vertex 0 and
 * velocities FP32, the inside test runs in FP32 and is redone with the
 * reference's FP64 weights when the smallest weight is within 1e-5 of zero,
 * and the density still accumulates in FP64.  In the mixed form a particle
 * whose FP64 weights all lie within 1e-10 of [0, 1] stays in its tet: the
 * reference's formula can put a point on a face shared by two tets outside
 * both, and its walk (src/meshes.h:75-100) would then never end.  Converts the
 * resident particles (holes removed first). */
int mp_set_particle_form(mp_ctx *ctx, int form);
/* Arithmetic of the mixed-form Newton factorization:
 *   MP_MIXED_TF32    one TF32 product per term (more FP64 refinement solves);
 *   MP_MIXED_FP16    the trailing updates on FP16 copies of their operands,
 *                    scaled by powers of two: the same 11 significant bits as
 *                    TF32 (rounded to nearest) at half the operand bytes and
 *                    twice the tensor rate; if a scaled operand would overflow
 *                    FP16 the factorization is redone with TF32 operands;
 *   MP_MIXED_TF32X3  hi/lo split, three TF32 products a term (about FP32
 *                    accuracy, fewer refinement solves);
 *   MP_MIXED_AUTO    the default: TF32X3 below MP_MIXED_FP16_FROM unknowns,
 *                    where the refinement solves cost more than the trailing
 *                    update saves, FP16 from there on.
 * Either way the solve is refined in FP64 to the same tolerance.  No
 * reference counterpart: the reference's dsysv_ call (src/FESolver.cpp:528-558)
 * is FP64 throughout. */
#define MP_MIXED_FP16_FROM 16384
int mp_set_mixed_factor(mp_ctx *ctx, int mode);
/* Particle IDs (16 B per particle-step of traffic) are needed only to restore
 * injection order after tet re-sorting; without sorting the stable removal
 * keeps the reference's order by itself.  With IDs off and sorting on,
 * downloads come in storage order.  Default on. */
int mp_set_track_ids(mp_ctx *ctx, int on);
/* Device address and length (elements) of a context buffer named by MP_VEC_*
 * (FP64 vectors), for zero-copy interop on the context's stream: e.g. an
 * all-reduce of the node density across ranks between mp_push_scatter and
 * mp_compute_phi.  No counterpart in the reference (single process). */
int mp_device_buffer(mp_ctx *ctx, int which, void **ptr, int64_t *len);
/* Kernels this context has launched since creation (for launch accounting). */
int mp_kernel_launches(mp_ctx *ctx, int64_t *n);
/* Device time of kernel classes, for roofline accounting (no reference
 * counterpart; the reference's trace.csv times host functions, src/trace.cpp).
 * While on, CUDA events bracket every launch of the classes below and each
 * call reads them after its own synchronisation; any call resets the clocks.
 * on = 0: off; 1: every class; otherwise a mask of (1 << MP_KT_*) bits (the
 * diagonal-block and panel classes launch hundreds of small kernels a step,
 * whose event records slow the host's launch stream, so a timed run leaves
 * them out).  work: algorithmic bytes for MP_KT_PUSH ((particles before + after
 * the push) x the form's bytes per particle, 52 FP64 / 28 mixed), algorithmic
 * flops for MP_KT_UPDATE (2 per multiply-add of the trailing update's lower
 * triangle; the 3xTF32 split issues three tensor-core products per term and
 * counts once), 0 for the latency-bound classes. */
enum { MP_KT_PUSH = 0,    /* the push + walk + scatter kernel */
       MP_KT_UPDATE = 1,  /* trailing updates of the LDL^T: tcgen05 (mixed) or register-tiled FP64 */
       MP_KT_DIAG = 2,    /* diagonal-block factorizations */
       MP_KT_PANEL = 3,   /* panels, in-panel column updates and operand splits */
       MP_KT_TRSV = 4     /* triangular solves */ };
int mp_set_kernel_timing(mp_ctx *ctx, int on);
int mp_kernel_timing(mp_ctx *ctx, int kernel_class, int64_t *launches, double *ms, double *work);

/* ---- particles ---------------------------------------------------------------- */
int mp_particles_reserve(mp_ctx *ctx, int64_t capacity);
/* Appends n particles from host memory (strided like the reference's Particle,
 * 88 B).  If rewind != 0 the device applies InjectIons' half-step velocity
 * rewind with the current device E field: vel -= (q_over_m*ef[cell])*half_dt
 * (src/mini-pic.cpp:253-257).  New particles get consecutive IDs. */
int mp_particles_append(mp_ctx *ctx, int64_t n,
                        const double *pos, int64_t pos_stride,
                        const double *vel, int64_t vel_stride,
                        const int32_t *cell, int64_t cell_stride,
                        int rewind, double q_over_m, double half_dt);
/* Appends from device memory: SoA arrays pos[3][n], vel[3][n], cell[n]. */
int mp_particles_append_device(mp_ctx *ctx, int64_t n, const double *pos_soa, const double *vel_soa,
                               const int32_t *cell, int rewind, double q_over_m, double half_dt);
int mp_particles_count(mp_ctx *ctx, int64_t *n);
/* Copies all particles to host memory, strided; any output may be NULL.  lc
 * gets the barycentric weights in the current tet (recomputed exactly as the
 * walk computes them).  order = MP_ORDER_ID returns injection order. */
int mp_particles_download(mp_ctx *ctx, int64_t n_max,
                          double *pos, int64_t pos_stride,
                          double *vel, int64_t vel_stride,
                          int32_t *cell, int64_t cell_stride,
                          double *lc, int64_t lc_stride,
                          int64_t *id, int order);
int mp_particles_clear(mp_ctx *ctx);

/* ---- MoveParticles -------------------------------------------------------------- */
/* One push: E gather + kick + drift + tet walk + density scatter for every
 * particle, stable removal of the particles that left the domain, and the
 * normalisation den[n] *= spwt / node_volume[n].  The density stays on the
 * device for mp_compute_phi; den_out (host, nullable) receives a copy. */
int mp_push_scatter(mp_ctx *ctx, double q_over_m, double dt, double spwt,
                    double *den_out, mp_step_stats *stats);
int mp_density_download(mp_ctx *ctx, double *den);
int mp_sort_by_tet(mp_ctx *ctx);

/* Allocation-free push for callers that cannot allocate device memory: code
 * whose GPU memory is all handed out by another allocator or runtime, and code
 * on a latency-critical path where cudaMalloc is not allowed because it can
 * synchronise the whole device.  No counterpart in the reference: it is the
 * device body of MoveParticles (src/mini-pic.cpp:287-308, walk
 * src/meshes.h:75-100) run on caller-owned device buffers in the reference's
 * own record layouts, plus the stable removal of the particles that left the
 * domain.
 *   particles_in/out  n Particle records (88 B: pos[3], vel[3], lc[4], cell);
 *                     out receives the kept particles in order with their
 *                     weights; out may equal in
 *   tetra             n_tets Tetra records (168 B) as LoadVolumeMesh builds them
 *   ef, den           [n_tets][3] field; [n_nodes] density, zeroed by the call
 *                     then summed (not yet multiplied by spwt/node volume)
 *   stream            a cudaStream_t (NULL: the default stream); the call
 *                     returns after the stream has finished its work
 *   n_out             host: number of particles kept
 * All pointers except n_out are device pointers on the current device.  The
 * kernel's scratch (look-back words of the compaction and three counters,
 * 262,208 B) is a fixed device array of the library, held on every GPU that
 * loads it until exit and shared by every call: n above 8,388,608 returns
 * MP_ERR_LIMIT; calls that overlap on the GPU race on the scratch and must be
 * serialised; the first call on a device looks the array up with that device
 * current and should come before any stream capture.  Walk limit 4096 hops
 * (MP_ERR_WALK_LIMIT).  Every index in the caller's records is checked before
 * use: a particle whose cell is outside [0, n_tets) (the reference's removed
 * state cell_index = -1 included), or whose walk meets a neighbour index
 * >= n_tets or a node index outside [0, n_nodes), stops there, adds nothing to
 * den, is written out as it stands and the call returns MP_ERR_ARG.  After
 * MP_ERR_TIMEOUT the contents of particles_out (and of particles_in when it is
 * the same buffer) are undefined. */
int mp_push_particles_noalloc(const void *particles_in, void *particles_out, int64_t n,
                              const void *tetra, int32_t n_tets, const double *ef, double *den,
                              int32_t n_nodes, double q_over_m, double dt, void *stream, int64_t *n_out);

/* ---- field solve ------------------------------------------------------------------ */
int mp_fe_setup(mp_ctx *ctx, const mp_fe_desc *fe);
/* Chooses the storage of K (MP_FE_STORAGE_*); call before mp_fe_setup. */
int mp_set_fe_storage(mp_ctx *ctx, int storage);
/* Conjugate-gradient stop: ||G - J y||_2 <= rtol ||G||_2 (default 1e-12) within
 * max_iterations (default 20000; MP_ERR_NOT_CONVERGED past it). */
int mp_set_sparse_solver(mp_ctx *ctx, double rtol, int32_t max_iterations);
/* The sparse K as CSR (columns ascending): with row_ptr, col and val all NULL
 * only *nnz is written; else row_ptr[neq + 1], col[nnz], val[nnz]. */
int mp_fe_sparse_matrix(mp_ctx *ctx, int64_t *nnz, int64_t *row_ptr, int32_t *col, double *val);
int mp_fe_upload(mp_ctx *ctx, int which, const double *values);
int mp_fe_download(mp_ctx *ctx, int which, double *out);
/* FESolver::computePhi: ion_den (host, nullable = the device density of the last
 * push) -> Newton step(s) by `method` -> uh = g + d. */
int mp_compute_phi(mp_ctx *ctx, const double *ion_den, int method, int form, mp_newton_stats *stats);
int mp_fe_build_f1(mp_ctx *ctx, const double *ion_den);
int mp_fe_residual(mp_ctx *ctx);
int mp_fe_build_j(mp_ctx *ctx, int method);
/* Solves J y = G (G from mp_fe_residual, or b if non-NULL); y stays on the device
 * (MP_VEC_Y).  method MP_METHOD_GAUSS_SEIDEL, MP_METHOD_LAPACK or MP_METHOD_SPARSE_CG.
 * Gauss-Seidel that ends its sweeps with sqrt(sum r^2)/neq >= 1e-4 (solveLinear,
 * src/FESolver.cpp:561-601) returns MP_ERR_NOT_CONVERGED with y holding the last
 * iterate; inside mp_compute_phi the step goes on, as the reference's does, and
 * the failure is counted in mp_newton_stats.linear_failures. */
int mp_fe_solve_linear(mp_ctx *ctx, int method, int form, const double *b, mp_newton_stats *stats);
/* Sweep limit of Gauss-Seidel (default 10000, the reference's). */
int mp_set_gs_max_sweeps(mp_ctx *ctx, int32_t sweeps);
/* FESolver::updateEf from the device uh (or uh_host if non-NULL). */
int mp_update_ef(mp_ctx *ctx, const double *uh_host);
int mp_field_download(mp_ctx *ctx, double *d, double *uh, double *ef);

/* ---- VTK output ---------------------------------------------------------------------- */
/* OutputMesh (src/meshes.cpp:358-447): writes mesh_<ts+1, 4 digits>.vtu into
 * `dir` (NULL or "" = the current directory) with the reference's ASCII text
 * byte for byte, from the context's uh, ef and node density (the last push's)
 * and the caller's node types (node_type_stride bytes apart; 40 for an array
 * of the reference's Node).  Asynchronous: the call copies the arrays to
 * pinned host memory on the context's stream, opens the file (MP_ERR_ARG if it
 * cannot, where the reference exits) and returns; a writer thread formats and
 * writes.  A later output call, mp_output_wait or mp_destroy joins it. */
int mp_output_mesh(mp_ctx *ctx, int32_t ts, const char *dir, const int32_t *node_type, int64_t node_type_stride);
/* OutputParticles (src/particles.cpp:21-45): the live particles' positions in
 * the reference's order, written to `path` (the reference's is
 * "particles.vtp") by the writer thread. */
int mp_output_particles(mp_ctx *ctx, const char *path);
/* Joins the writer; returns its status (MP_ERR_ARG if the write failed). */
int mp_output_wait(mp_ctx *ctx);

/* ---- host-side setup helpers (no device needed) ----------------------------------- */
/* LoadVolumeMesh's geometry (src/meshes.cpp:80-262) from node positions in metres
 * and 0-based tet connectivity.  con is fixed in place for negative volumes.
 * Outputs: volume[n_tets], alpha/beta/gamma/delta[n_tets][4], cell_con[n_tets][4],
 * node_volume[n_nodes], node_open[n_nodes] (1 where the reference marks OPEN). */
int mp_mesh_geometry(int32_t n_nodes, const double *node_pos, int32_t n_tets, int32_t *con,
                     double *volume, double *alpha, double *beta, double *gamma, double *delta,
                     int32_t *cell_con, double *node_volume, int32_t *node_open);
/* FESolver ctor bookkeeping (src/FESolver.cpp:48-127): ID from node types
 * (0 NORMAL, 1 OPEN, 2 INLET, 3 FIXED), NX and detJ.  Returns neq in *neq. */
int mp_fe_geometry(int32_t n_nodes, const double *node_pos, const int32_t *node_type,
                   int32_t n_tets, const int32_t *con, int32_t *ID, double *nx, double *detJ, int32_t *neq);
/* LoadSurfaceMesh's inlet face data (src/meshes.cpp:290-353): owning tet, u, v,
 * unit normal and area of each inlet triangle (0-based node ids). */
int mp_inlet_faces(int32_t n_nodes, const double *node_pos, int32_t n_tets, const int32_t *con,
                   int32_t n_faces, const int32_t *face_con, int invert_normals,
                   int32_t *cell_con, double *u, double *v, double *normal, double *area);

/* The three helpers above computed on device `device` (host arrays in and
 * out; the same outputs bit for bit).  Face neighbours and inlet faces' tets
 * come from the tets' faces sorted by node triple instead of the reference's
 * scans over tets (src/meshes.cpp:180-227, 306-326).  MP_ERR_ARG for an index
 * out of range, a face held by three tets, or an inlet face held by no tet or
 * by two (where the reference exits); at most 2^29 tets. */
int mp_mesh_geometry_device(int device, int32_t n_nodes, const double *node_pos, int32_t n_tets, int32_t *con,
                            double *volume, double *alpha, double *beta, double *gamma, double *delta,
                            int32_t *cell_con, double *node_volume, int32_t *node_open);
int mp_inlet_faces_device(int device, int32_t n_nodes, const double *node_pos, int32_t n_tets,
                          const int32_t *con, int32_t n_faces, const int32_t *face_con, int invert_normals,
                          int32_t *cell_con, double *u, double *v, double *normal, double *area);
int mp_fe_geometry_device(int device, int32_t n_nodes, const double *node_pos, const int32_t *node_type,
                          int32_t n_tets, const int32_t *con, int32_t *ID, double *nx, double *detJ,
                          int32_t *neq);

/* InjectIons (src/mini-pic.cpp:208-265) with the reference's RNG stream
 * (std::mt19937 seeded 0, uniform_real_distribution<double>(0,1)). */
typedef struct mp_injector mp_injector;
int mp_injector_create(int32_t n_faces, const int32_t *face_con, const double *u, const double *v,
                       const double *normal, const double *area, const int32_t *cell_con,
                       const double *node_pos, uint32_t seed, mp_injector **out);
int mp_injector_destroy(mp_injector *inj);
/* Samples one step's particles into caller buffers (capacity max_n, SoA-strided
 * like mp_particles_append).  The velocity rewind is not applied (pass rewind=1
 * to mp_particles_append).  *n_out = particles written. */
int mp_injector_sample(mp_injector *inj, double plasma_den, double ion_velocity, double dt, double spwt,
                       int64_t max_n, double *pos, int64_t pos_stride, double *vel, int64_t vel_stride,
                       int32_t *cell, int64_t cell_stride, int64_t *n_out);
int mp_injector_count(mp_injector *inj, double plasma_den, double ion_velocity, double dt, double spwt,
                      int64_t *n_next);
int mp_injector_get_rem(mp_injector *inj, double *rem);
/* InjectIons on the device (src/mini-pic.cpp:208-265): the reference's per-face
 * counts, with the injector's shared remainder carried exactly as
 * mp_injector_sample carries it, and positions (uniform on each inlet
 * triangle, the reference's a+b>1 fold) and velocities (normal*ion_velocity
 * plus a Maxwellian thermal part of standard deviation thermal_sigma per
 * component; 0 = the reference's cold beam) drawn on the device with
 * Philox4x32-10 keyed by seed at counter (particle, step) instead of the
 * reference's mt19937 stream.  The particles are appended with the half-step
 * rewind in the current device field (q_over_m, dt/2).  No particle crosses
 * the host; *n_out (nullable) = particles injected. */
int mp_inject_device(mp_ctx *ctx, mp_injector *inj, double plasma_den, double ion_velocity, double dt, double spwt,
                     double thermal_sigma, double q_over_m, uint64_t seed, uint64_t step, int64_t *n_out);
int mp_injector_set_rem(mp_injector *inj, double rem);

/* ---- adjoint of K push + scatter steps ---------------------------------------
 * phi (node potential, uh's layout) is held for K steps, so ef = updateEf(phi)
 * (src/FESolver.cpp:622-636) is fixed and each particle moves on its own:
 *   injected at step k0: v = inlet_dir*v_drift + v_th - (q_over_m*ef[c])*(0.5*dt)
 *                        (src/mini-pic.cpp:239-257; v_th = 0 is the reference's cold beam)
 *   each step:           the MoveParticles kernel body and XtoLtet walk
 *                        (src/mini-pic.cpp:287-308, src/meshes.h:75-100)
 * Outputs: den, the last step's node density normalised by spwt/Vnode
 * (src/mini-pic.cpp:319), and flux, the wall energy flux
 *   F = sum over particles leaving through a wall face of spwt*(0.5*mass)*|v|^2
 * (v after the exit step's kick; a wall face is a boundary face whose three
 * nodes have wall_nodes[n] != 0).  Derivatives treat the walk as piecewise
 * fixed (cells and exits held).  Particles keep their slots for the K steps;
 * the forward stores each slot's state every checkpoint_every steps and the
 * reverse recomputes each segment from its checkpoint.
 * Vector arguments (phi, den, bars, tangents, particle arrays) may be host or
 * device memory. */
enum { MP_ADJ_WALK = 0,    /* walk with XtoLtet (records the path if asked) */
       MP_ADJ_PINNED = 1   /* replay the recorded path: the piecewise-fixed model itself */ };
typedef struct {
    int64_t slots;        /* particles carried: initial population + injections */
    int64_t alive;        /* inside the domain after the last step */
    int64_t wall_exits;   /* left through a wall face */
    int64_t other_exits;  /* left through another boundary face */
    double flux;          /* wall energy flux F [J] */
    float ms;             /* device time of the forward */
} mp_adjoint_stats;
/* steps K >= 1; checkpoint_every in [1, 32]; inlet_dir[3] is the inlet face
 * normal of InjectIons; nx [n_tets][4][3] (FESolver::NX) or NULL for the FE
 * setup's; record_path keeps the walked cells for MP_ADJ_PINNED replays. */
int mp_adjoint_setup(mp_ctx *ctx, int32_t steps, int32_t checkpoint_every, double q_over_m, double mass,
                     double dt, double spwt, const double *inlet_dir, const uint8_t *wall_nodes, const double *nx,
                     int record_path);
/* Adds n particles entering at first_step (0 = the initial population).
 * pos/vel packed [n][3]; injected != 0: vel is the thermal part v_th and the
 * drift and rewind are applied as above; injected == 0: vel is the velocity. */
int mp_adjoint_add_particles(mp_ctx *ctx, int32_t first_step, int injected, int64_t n, const double *pos,
                             const double *vel, const int32_t *cell);
/* Runs the K steps: den_out [n_nodes] (nullable), stats (nullable).  Keeps the
 * tape (checkpoints, outcomes) for mp_adjoint_backward / mp_adjoint_tangent. */
int mp_adjoint_forward(mp_ctx *ctx, const double *phi, double v_drift, int mode, double *den_out,
                       mp_adjoint_stats *st);
int mp_adjoint_flux(mp_ctx *ctx, double *flux);
/* Vector-Jacobian product at the last forward: phi_bar = (dden/dphi)^T den_bar
 * + (dF/dphi)^T flux_bar, *v_drift_bar likewise.  den_bar NULL means zero. */
int mp_adjoint_backward(mp_ctx *ctx, const double *den_bar, double flux_bar, double *phi_bar, double *v_drift_bar);
/* Jacobian-vector product at the last forward: dden = dden/dphi dphi + dden/dvd dv_drift,
 * *dflux likewise (the tangents a coupled ion-phi Newton-Krylov solve uses). */
int mp_adjoint_tangent(mp_ctx *ctx, const double *dphi, double dv_drift, double *dden, double *dflux);

#ifdef __cplusplus
}
#endif
#endif /* MINIPIC_CUDA_H */
