/* Test infrastructure: oracle.c, a plain-C restatement of the reference's
 * algorithm for the hot path.  Used only by tests, smoke() and bench.py's CPU
 * baseline leg, as the checker; never linked by the product.
 *
 * Arrays are packed: pos/vel [n][3], lc [n][4], tets' con/alpha/.../cell_con
 * [n_tets][4], NX [n_tets][4][3], dense matrices row-major [neq][neq]. */
#ifndef MINIPIC_ORACLE_H
#define MINIPIC_ORACLE_H
#include <stdint.h>

typedef struct {
    uint32_t mt[624];
    int idx;
} or_mt;

void or_mt_seed(or_mt *g, uint32_t seed);
uint32_t or_mt_next(or_mt *g);
double or_rnd(or_mt *g);

long or_inject(or_mt *g, double *rem, int n_faces, const int *face_con, const double *u, const double *v,
               const double *normal, const double *area, const int *face_cell, const double *node_pos,
               double plasma_den, double ion_velocity, double dt, double spwt, long max_n, double *pos,
               double *vel, int *cell);
void or_rewind(long n, double *vel, const int *cell, const double *ef, double q_over_m, double half_dt);

long or_push(long n, double *pos, double *vel, int *cell, double *lc, const int *con, const double *volume,
             const double *alpha, const double *beta, const double *gamma, const double *delta,
             const int *cell_con, const double *ef, double q_over_m, double dt, double *den, int n_nodes,
             long *hops_out);
long or_compact(long n, double *pos, double *vel, int *cell, int64_t *id);
void or_normalise(int n_nodes, double *den, const double *node_volume, double spwt);

void or_update_ef(int n_tets, const int *con, const double *nx, const double *uh, double *ef);
void or_build_f1(int n_nodes, int n_tets, int neq, const int *ID, const int *con, const double *detJ,
                 const double *ion_den, const double *d, double n0, double phi0, double kTe, double *F1);
void or_build_fp(int n_tets, int neq, const int *ID, const int *con, const double *detJ, const double *d,
                 double n0, double phi0, double kTe, double *FP);
void or_residual(int neq, const double *K, const double *d, const double *F0, const double *F1, double *G);
void or_build_j(int neq, const double *K, const double *FP, double *J);
int or_gauss_seidel(int neq, const double *A, const double *b, double *x, double *L2_out);
int or_solve_dense(int neq, double *A, double *b);
void or_assemble(int n_tets, int neq, const int *ID, const int *con, const double *nx, const double *detJ,
                 const double *g, double *K, double *F0);
void or_uh(int n_nodes, const int *ID, const double *g, const double *d, double *uh);

#endif
