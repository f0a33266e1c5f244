/* Test infrastructure: plain-C restatement of the reference's algorithm for the
 * mini-pic hot path (AD1641/mini-fem-pic-main).  Each function cites the
 * reference lines it follows and keeps their expression order; the file is
 * compiled with -ffp-contract=off so no FMA contraction changes a rounding.
 * It is pinned against the reference's own compiled code (oracle/_ref) and
 * against the committed fixtures in tests/golden/.  Only tests, smoke() and
 * bench.py's CPU-baseline leg use it, as the checker. */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double QE = 1.602e-19;       /* src/FESolver.h:19 */
static const double EPS0 = 8.8541878e-12; /* src/FESolver.h:18 */

/* ---- RNG: std::mt19937 (Matsumoto & Nishimura 1998, the C++ standard's
 * parameters) and libstdc++'s generate_canonical<double,53> over it, which is
 * what uniform_real_distribution<double>(0,1) returns (src/maths.cpp:17-19). */
void or_mt_seed(or_mt *g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; i++) g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

uint32_t or_mt_next(or_mt *g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; i++) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

double or_rnd(or_mt *g) {
    /* two 32-bit draws, low word first: (r0 + r1*2^32) / 2^64, clamped below 1 */
    double sum = 0.0, tmp = 1.0;
    for (int k = 0; k < 2; k++) {
        sum += (double)or_mt_next(g) * tmp;
        tmp *= 4294967296.0;
    }
    double r = sum / tmp;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

/* ---- InjectIons without the velocity rewind, src/mini-pic.cpp:212-262 ---- */
long or_inject(or_mt *g, double *rem, int n_faces, const int *face_con, const double *u, const double *v,
               const double *normal, const double *area, const int *face_cell, const double *node_pos,
               double plasma_den, double ion_velocity, double dt, double spwt, long max_n, double *pos,
               double *vel, int *cell) {
    long k = 0;
    for (int f = 0; f < n_faces; f++) {
        double num_per_sec = plasma_den * ion_velocity * area[f];
        double num_real = num_per_sec * dt;
        double fnum_mp = num_real / spwt + *rem;
        int num_mp = (int)fnum_mp;
        *rem = fnum_mp - num_mp;
        const double *p0 = node_pos + 3 * (long)face_con[3 * f];
        for (int p = 0; p < num_mp; p++) {
            double a = or_rnd(g);
            double b = or_rnd(g);
            if ((a + b) > 1) {
                a = 1 - a;
                b = 1 - b;
            }
            if (k < max_n) {
                for (int i = 0; i < 3; i++) {
                    pos[3 * k + i] = a * u[3 * f + i] + b * v[3 * f + i] + p0[i];
                    vel[3 * k + i] = normal[3 * f + i] * ion_velocity;
                }
                cell[k] = face_cell[f];
            }
            k++;
        }
    }
    return k;
}

/* vel -= charge/mass*ef*(0.5*dt), src/mini-pic.cpp:253-257 */
void or_rewind(long n, double *vel, const int *cell, const double *ef, double q_over_m, double half_dt) {
    for (long p = 0; p < n; p++)
        for (int i = 0; i < 3; i++) vel[3 * p + i] -= q_over_m * ef[3 * (long)cell[p] + i] * half_dt;
}

/* ---- XtoLtet, src/meshes.h:75-100 --------------------------------------------- */
static int xtoltet(const double *x, int *cellp, double *lc, const double *volume, const double *alpha,
                   const double *beta, const double *gamma, const double *delta, const int *cell_con, long *hops) {
    for (;;) {
        int c = *cellp;
        int inside = 1;
        for (int i = 0; i < 4; i++) {
            lc[i] = (1.0 / 6.0) *
                    (alpha[4 * c + i] - x[0] * beta[4 * c + i] + x[1] * gamma[4 * c + i] - x[2] * delta[4 * c + i]) /
                    volume[c];
            if (lc[i] < 0 || lc[i] > 1.0) inside = 0;
        }
        if (inside) return 1;
        int min_i = 0;
        double min_lc = lc[0];
        for (int i = 1; i < 4; i++)
            if (lc[i] < min_lc) {
                min_lc = lc[i];
                min_i = i;
            }
        if (cell_con[4 * c + min_i] < 0) return 0;
        *cellp = cell_con[4 * c + min_i];
        (*hops)++;
    }
}

/* ---- MoveParticles' kernel body, src/mini-pic.cpp:287-308, particles in order.
 * den is zeroed first (src/mini-pic.cpp:277).  Exits get cell -1. ---------- */
long or_push(long n, double *pos, double *vel, int *cell, double *lc, const int *con, const double *volume,
             const double *alpha, const double *beta, const double *gamma, const double *delta,
             const int *cell_con, const double *ef, double q_over_m, double dt, double *den, int n_nodes,
             long *hops_out) {
    long removed = 0, hops = 0;
    for (int k = 0; k < n_nodes; k++) den[k] = 0.0;
    for (long p = 0; p < n; p++) {
        double *x = pos + 3 * p, *v = vel + 3 * p;
        double l[4];
        for (int i = 0; i < 3; i++) v[i] += q_over_m * ef[3 * (long)cell[p] + i] * dt;
        for (int i = 0; i < 3; i++) x[i] += v[i] * dt;
        if (xtoltet(x, &cell[p], l, volume, alpha, beta, gamma, delta, cell_con, &hops)) {
            for (int q = 0; q < 4; q++) den[con[4 * (long)cell[p] + q]] += l[q];
        } else {
            cell[p] = -1;
            removed++;
        }
        if (lc)
            for (int q = 0; q < 4; q++) lc[4 * p + q] = l[q];
    }
    if (hops_out) *hops_out = hops;
    return removed;
}

/* std::erase_if(cell_index < 0), src/mini-pic.cpp:316: stable, in place. */
long or_compact(long n, double *pos, double *vel, int *cell, int64_t *id) {
    long w = 0;
    for (long p = 0; p < n; p++) {
        if (cell[p] < 0) continue;
        if (w != p) {
            memmove(pos + 3 * w, pos + 3 * p, 3 * sizeof(double));
            memmove(vel + 3 * w, vel + 3 * p, 3 * sizeof(double));
            cell[w] = cell[p];
            if (id) id[w] = id[p];
        }
        w++;
    }
    return w;
}

/* den[n] *= spwt/node.volume, src/mini-pic.cpp:319 */
void or_normalise(int n_nodes, double *den, const double *node_volume, double spwt) {
    for (int k = 0; k < n_nodes; k++) den[k] *= spwt / node_volume[k];
}

/* ---- FESolver::updateEf, src/FESolver.cpp:622-636 ---- */
void or_update_ef(int n_tets, const int *con, const double *nx, const double *uh, double *ef) {
    for (int e = 0; e < n_tets; e++) {
        for (int d = 0; d < 3; d++) ef[3 * e + d] = 0;
        for (int a = 0; a < 4; a++) {
            int A = con[4 * e + a];
            for (int d = 0; d < 3; d++) ef[3 * e + d] -= nx[12 * e + 3 * a + d] * uh[A];
        }
    }
}

/* quadrature points, src/FESolver.cpp:114-117 and evalNa 188-196 */
static void na_table(double Na[4][8]) {
    double l[2] = {-sqrt(1.0 / 3.0), sqrt(1.0 / 3.0)};
    int p = 0;
    for (int k = 0; k < 2; k++)
        for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
                double xi = 0.5 * (l[i] + 1), eta = 0.5 * (l[j] + 1), zeta = 0.5 * (l[k] + 1);
                Na[0][p] = xi;
                Na[1][p] = eta;
                Na[2][p] = zeta;
                Na[3][p] = 1 - xi - eta - zeta;
                p++;
            }
}

/* element loop of buildF1Vector / buildJmatrix: out[A] += (sum_p t[A]*Na*detJ)*(1/8) */
static void element_terms(int n_tets, const int *ID, const int *con, const double *detJ, const double *t,
                          double *out) {
    double Na[4][8];
    na_table(Na);
    for (int e = 0; e < n_tets; e++)
        for (int a = 0; a < 4; a++) {
            int A = ID[con[4 * e + a]];
            if (A < 0) continue;
            double ff = 0;
            for (int p = 0; p < 8; p++) ff += t[A] * Na[a][p] * detJ[e] * 1.0 * 1.0 * 1.0;
            ff *= (1.0 / 8.0);
            out[A] += ff;
        }
}

/* FESolver::buildF1Vector, src/FESolver.cpp:488-526 (F1 accumulates) */
void or_build_f1(int n_nodes, int n_tets, int neq, const int *ID, const int *con, const double *detJ,
                 const double *ion_den, const double *d, double n0, double phi0, double kTe, double *F1) {
    double *f = (double *)calloc((size_t)neq + 1, sizeof(double));
    for (int n = 0; n < n_nodes; n++) {
        int A = ID[n];
        if (A < 0) continue;
        f[A] = (QE / EPS0) * (ion_den[n] + n0 * exp((d[A] - phi0) / kTe));
    }
    element_terms(n_tets, ID, con, detJ, f, F1);
    free(f);
}

/* FP of FESolver::buildJmatrix, src/FESolver.cpp:367-424 */
void or_build_fp(int n_tets, int neq, const int *ID, const int *con, const double *detJ, const double *d,
                 double n0, double phi0, double kTe, double *FP) {
    double *fp = (double *)calloc((size_t)neq + 1, sizeof(double));
    for (int n = 0; n < neq; n++) fp[n] = -QE / EPS0 * n0 * exp((d[n] - phi0) / kTe) * (1 / kTe);
    for (int n = 0; n < neq; n++) FP[n] = 0;
    element_terms(n_tets, ID, con, detJ, fp, FP);
    free(fp);
}

/* J = K; J[u][u] -= FP[u], src/FESolver.cpp:378-428 */
void or_build_j(int neq, const double *K, const double *FP, double *J) {
    memcpy(J, K, sizeof(double) * (size_t)neq * neq);
    for (int u = 0; u < neq; u++) J[(size_t)u * neq + u] -= FP[u];
}

/* G = K d; G -= F0; G -= F1, src/FESolver.cpp:333-335 with maths.cpp:60-73 */
void or_residual(int neq, const double *K, const double *d, const double *F0, const double *F1, double *G) {
    for (int i = 0; i < neq; i++) {
        double y = 0;
        for (int j = 0; j < neq; j++) y += K[(size_t)i * neq + j] * d[j];
        G[i] = y;
    }
    for (int i = 0; i < neq; i++) G[i] = G[i] - F0[i];
    for (int i = 0; i < neq; i++) G[i] = G[i] - F1[i];
}

/* FESolver::solveLinear, src/FESolver.cpp:561-601.  Returns sweeps done. */
int or_gauss_seidel(int neq, const double *A, const double *b, double *x, double *L2_out) {
    const double tol = 1e-4;
    double L2 = 0;
    int it;
    for (it = 0; it < 10000; it++) {
        for (int u = 0; u < neq; u++) {
            if (fabs(A[(size_t)u * neq + u]) < 1e-12) continue;
            double sum = 0;
            for (int v = 0; v < neq; v++) {
                if (u == v) continue;
                sum += A[(size_t)u * neq + v] * x[v];
            }
            x[u] = (b[u] - sum) / A[(size_t)u * neq + u];
        }
        if (it % 25 == 0) {
            double L = 0;
            for (int u = 0; u < neq; u++) {
                double sum = 0;
                for (int v = 0; v < neq; v++) sum += A[(size_t)u * neq + v] * x[v];
                double r = b[u] - sum;
                L += r * r;
            }
            L2 = sqrt(L) / neq;
            if (L2 < tol) break;
        }
    }
    if (L2_out) *L2_out = L2;
    return it;
}

/* Dense solve A x = b (b overwritten with x) by Gaussian elimination with
 * partial pivoting: stands in for LAPACK's dsysv_ (src/FESolver.cpp:550), whose
 * result it matches to rounding for the nonsingular J.  Returns 0, or k+1 at a
 * zero pivot. */
int or_solve_dense(int n, double *A, double *b) {
    for (int k = 0; k < n; k++) {
        int piv = k;
        double best = fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(A[(size_t)i * n + k]) > best) {
                best = fabs(A[(size_t)i * n + k]);
                piv = i;
            }
        if (best == 0.0) return k + 1;
        if (piv != k) {
            for (int j = 0; j < n; j++) {
                double t = A[(size_t)k * n + j];
                A[(size_t)k * n + j] = A[(size_t)piv * n + j];
                A[(size_t)piv * n + j] = t;
            }
            double t = b[k];
            b[k] = b[piv];
            b[piv] = t;
        }
        for (int i = k + 1; i < n; i++) {
            double l = A[(size_t)i * n + k] / A[(size_t)k * n + k];
            if (l == 0.0) continue;
            for (int j = k; j < n; j++) A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
            b[i] -= l * b[k];
        }
    }
    for (int k = n - 1; k >= 0; k--) {
        double s = b[k];
        for (int j = k + 1; j < n; j++) s -= A[(size_t)k * n + j] * b[j];
        b[k] = s / A[(size_t)k * n + k];
    }
    return 0;
}

/* FESolver::startAssembly + preAssembly, src/FESolver.cpp:155-163, 434-485 */
void or_assemble(int n_tets, int neq, const int *ID, const int *con, const double *nx, const double *detJ,
                 const double *g, double *K, double *F0) {
    memset(K, 0, sizeof(double) * (size_t)neq * neq);
    memset(F0, 0, sizeof(double) * (size_t)neq);
    for (int e = 0; e < n_tets; e++) {
        double ke[4][4];
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                ke[a][b] = 0;
                for (int p = 0; p < 8; p++) {
                    double dot = 0;
                    for (int d = 0; d < 3; d++) dot += nx[12 * e + 3 * a + d] * nx[12 * e + 3 * b + d];
                    ke[a][b] += dot * detJ[e] * 1.0 * 1.0 * 1.0;
                }
            }
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                int P = ID[con[4 * e + a]], Q = ID[con[4 * e + b]];
                if (P < 0 || Q < 0) continue;
                K[(size_t)P * neq + Q] += ke[a][b];
            }
        for (int a = 0; a < 4; a++) {
            double fh = 0, fg = 0;
            for (int b = 0; b < 4; b++) fg -= ke[a][b] * g[con[4 * e + b]];
            double fe = fh + fg;
            int P = ID[con[4 * e + a]];
            if (P >= 0) F0[P] += fe;
        }
    }
}

/* uh = g (+ d on unknowns), src/FESolver.cpp:610-618 */
void or_uh(int n_nodes, const int *ID, const double *g, const double *d, double *uh) {
    for (int n = 0; n < n_nodes; n++) {
        uh[n] = g[n];
        if (ID[n] >= 0) uh[n] += d[ID[n]];
    }
}
