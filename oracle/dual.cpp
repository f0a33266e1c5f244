// Test infrastructure: the FP64 dual-number (forward-mode) build of the
// reference push, the checker of the adjoint's derivatives.  Used only by
// tests; never linked by the product.
//
// A restatement, in a number type carrying (value, tangent), of K steps of
//   InjectIons' velocity set-up and rewind   src/mini-pic.cpp:239-257
//   the MoveParticles kernel body            src/mini-pic.cpp:287-308
//   XtoLtet                                  src/meshes.h:75-100
//   the density normalisation                src/mini-pic.cpp:319
//   FESolver::updateEf                       src/FESolver.cpp:622-636
// with phi held for the K steps.  The value part runs the reference's FP64
// operations in its order (no FMA: built with -ffp-contract=off), so it equals
// the reference push bit for bit; comparisons use the value part, so the
// walk is piecewise fixed exactly as the adjoint assumes.  Outputs are the
// last step's normalised node density and the wall energy flux
// F = sum over wall exits of spwt*(0.5*mass)*|v|^2, each with its tangent
// along (dphi, dv_drift).
#include <cstdint>
#include <vector>

namespace {

struct Dual {
    double v, d;
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual cst(double x) { return {x, 0.0}; }

struct Mesh {
    const int *con, *cell_con;
    const double *volume, *alpha, *beta, *gamma, *delta;
    const unsigned char *wall_nodes;
};

// XtoLtet: 1 inside (cell updated), 0 left the domain (exit face opposite *face)
int walk(const Mesh &m, int &cell, const Dual x[3], Dual lc[4], int *face) {
    for (long hops = 0; hops < (1l << 20); hops++) {
        const int t = cell;
        bool inside = true;
        for (int i = 0; i < 4; i++) {
            lc[i] = cst(1.0 / 6.0) * (cst(m.alpha[4 * t + i]) - x[0] * cst(m.beta[4 * t + i]) +
                                      x[1] * cst(m.gamma[4 * t + i]) - x[2] * cst(m.delta[4 * t + i])) /
                    cst(m.volume[t]);
            if (lc[i].v < 0 || lc[i].v > 1.0) inside = false;
        }
        if (inside) return 1;
        int min_i = 0;
        double min_lc = lc[0].v;
        for (int i = 1; i < 4; i++)
            if (lc[i].v < min_lc) {
                min_lc = lc[i].v;
                min_i = i;
            }
        if (m.cell_con[4 * t + min_i] < 0) {
            *face = min_i;
            return 0;
        }
        cell = m.cell_con[4 * t + min_i];
    }
    return -1;
}

bool wall_face(const Mesh &m, int t, int face) {
    for (int j = 0; j < 4; j++)
        if (j != face && !m.wall_nodes[m.con[4 * t + j]]) return false;
    return true;
}

}  // namespace

extern "C" {

// Returns 0, or -1 if a walk did not end.  Per particle outputs (nullable):
// kind (0 inside at the end, 1 left through a wall face, 2 left elsewhere),
// exit step (K if inside), final pos/vel [n][3] values, final cell, and a
// 64-bit FNV-1a hash of the cell at the end of every step (path identity).
int or_dual_ksteps(int n_tets, const int *con, const double *volume, const double *alpha, const double *beta,
                   const double *gamma, const double *delta, const int *cell_con, const double *nx, int n_nodes,
                   const double *node_volume, const unsigned char *wall_nodes, long n, const int *first,
                   const unsigned char *inj, const double *pos, const double *vel, const int *cell0, int K,
                   double qm, double mass, double dt, double spwt, const double *dir, const double *phi,
                   const double *dphi, double vd, double dvd, double *den, double *dden, double *flux,
                   double *dflux, int *kind_out, int *exit_out, double *pos_out, double *vel_out, int *cell_out,
                   uint64_t *path_out) {
    Mesh m{con, cell_con, volume, alpha, beta, gamma, delta, wall_nodes};
    // updateEf with the dual potential
    std::vector<Dual> ef(3 * (size_t)n_tets);
    for (int e = 0; e < n_tets; e++) {
        Dual f[3] = {cst(0), cst(0), cst(0)};
        for (int a = 0; a < 4; a++) {
            const int A = con[4 * e + a];
            const Dual u{phi[A], dphi ? dphi[A] : 0.0};
            for (int d = 0; d < 3; d++) f[d] = f[d] - cst(nx[12 * e + 3 * a + d]) * u;
        }
        for (int d = 0; d < 3; d++) ef[3 * e + d] = f[d];
    }
    std::vector<Dual> dn(n_nodes, cst(0));
    Dual F = cst(0);
    const Dual Vd{vd, dvd}, QM = cst(qm), DT = cst(dt);
    int rc = 0;
    for (long p = 0; p < n; p++) {
        Dual x[3], v[3];
        int c = cell0[p];
        for (int d = 0; d < 3; d++) {
            x[d] = cst(pos[3 * p + d]);
            v[d] = cst(vel[3 * p + d]);
        }
        if (inj[p])
            for (int d = 0; d < 3; d++) {
                v[d] = cst(dir[d]) * Vd + v[d];
                v[d] = v[d] - QM * ef[3 * c + d] * cst(0.5 * dt);
            }
        int kind = 0, ek = K;
        uint64_t hash = 1469598103934665603ull;
        Dual lc[4];
        for (int k = first[p]; k < K; k++) {
            for (int d = 0; d < 3; d++) v[d] = v[d] + QM * ef[3 * c + d] * DT;
            for (int d = 0; d < 3; d++) x[d] = x[d] + v[d] * DT;
            int face = 0;
            const int w = walk(m, c, x, lc, &face);
            hash = (hash ^ (uint64_t)(uint32_t)(w == 1 ? c : -1 - w)) * 1099511628211ull;
            if (w < 0) {
                rc = -1;
                kind = 2;
                ek = k;
                break;
            }
            if (w == 0) {
                kind = wall_face(m, c, face) ? 1 : 2;
                ek = k;
                break;
            }
        }
        if (kind == 1) F = F + cst(spwt) * (cst(0.5 * mass) * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        if (kind == 0)
            for (int i = 0; i < 4; i++) dn[con[4 * c + i]] = dn[con[4 * c + i]] + lc[i];
        if (kind_out) kind_out[p] = kind;
        if (exit_out) exit_out[p] = ek;
        if (cell_out) cell_out[p] = kind == 0 ? c : -1;
        if (path_out) path_out[p] = hash;
        for (int d = 0; d < 3; d++) {
            if (pos_out) pos_out[3 * p + d] = x[d].v;
            if (vel_out) vel_out[3 * p + d] = v[d].v;
        }
    }
    for (int i = 0; i < n_nodes; i++) {
        const Dual r = dn[i] * cst(spwt / node_volume[i]);
        if (den) den[i] = r.v;
        if (dden) dden[i] = r.d;
    }
    if (flux) *flux = F.v;
    if (dflux) *dflux = F.d;
    return rc;
}

}  // extern "C"
