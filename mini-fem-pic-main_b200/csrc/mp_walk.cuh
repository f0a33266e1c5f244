// The reference's barycentric coordinates and tet walk in FP64, bit for bit
// (every operation rounded on its own, in the reference's order: no FMA).
// Shared by the push kernels and the adjoint.
#pragma once

#include "mp_internal.h"

namespace mp {

constexpr double ONE_SIXTH = 1.0 / 6.0;

// Numerators q_i = (1.0/6.0)*(alpha_i - x*beta_i + y*gamma_i - z*delta_i) of
// the barycentric weights lambda_i = q_i/volume (src/meshes.h:84-85), in the
// reference's order, every operation rounded on its own.
__device__ __forceinline__ void numerators_fp64(const TetRec *__restrict__ t, double x, double y, double z,
                                                double q[4]) {
    const double2 *a2 = reinterpret_cast<const double2 *>(t->alpha);
    const double2 *b2 = reinterpret_cast<const double2 *>(t->beta);
    const double2 *g2 = reinterpret_cast<const double2 *>(t->gamma);
    const double2 *d2 = reinterpret_cast<const double2 *>(t->delta);
    double al[4], be[4], ga[4], de[4];
    double2 v;
    v = __ldg(a2); al[0] = v.x; al[1] = v.y; v = __ldg(a2 + 1); al[2] = v.x; al[3] = v.y;
    v = __ldg(b2); be[0] = v.x; be[1] = v.y; v = __ldg(b2 + 1); be[2] = v.x; be[3] = v.y;
    v = __ldg(g2); ga[0] = v.x; ga[1] = v.y; v = __ldg(g2 + 1); ga[2] = v.x; ga[3] = v.y;
    v = __ldg(d2); de[0] = v.x; de[1] = v.y; v = __ldg(d2 + 1); de[2] = v.x; de[3] = v.y;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        double w = __dsub_rn(al[i], __dmul_rn(x, be[i]));
        w = __dadd_rn(w, __dmul_rn(y, ga[i]));
        w = __dsub_rn(w, __dmul_rn(z, de[i]));
        q[i] = __dmul_rn(ONE_SIXTH, w);
    }
}

// The reference's lambda_i = q_i/volume, correctly rounded.
__device__ __forceinline__ void lambdas_fp64(const TetRec *__restrict__ t, double x, double y, double z,
                                             double lc[4]) {
    double q[4];
    numerators_fp64(t, x, y, z, q);
    const double vol = __ldg(&t->volume);
#pragma unroll
    for (int i = 0; i < 4; i++) lc[i] = __ddiv_rn(q[i], vol);
}

// XtoLtet (src/meshes.h:75-100) with a hop limit.  Returns 1 inside, 0 left the
// domain, -1 hop limit reached (cell is then the last tet visited).
//
// EXACT_CMP (every tet volume below 1): the inside test runs on the numerators,
// without the four divisions, and takes the same decisions.  With V > 0 and
// lambda = RN(q/V):
//   lambda < 0  <=>  q < 0   (q/V cannot round to -0 when V < 1: |q| >= 2^-1074)
//   lambda > 1  <=>  q > V   (if q > V then q >= V + ulp(V) > V(1 + 2^-53), the
//                             rounding midpoint above 1; if q <= V then q/V <= 1)
// and NaN compares false either way.  An inside particle's weights for the
// scatter are then q*RN(1/V) (within 2 ulp of lambda).  A particle outside its
// tet needs the exact lambdas for the hop (first minimum, strict <), so those
// are divided.
template <bool EXACT_CMP = false>
__device__ __forceinline__ int walk_fp64(const TetRec *__restrict__ tets, int &cell, double x, double y, double z,
                                         double lc[4], int limit, int &hops, int *exit_face = nullptr) {
    for (;;) {
        const TetRec *t = tets + cell;
        double q[4];
        numerators_fp64(t, x, y, z, q);
        const double vol = __ldg(&t->volume);
        if (EXACT_CMP) {
            bool inside = true;
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (q[i] < 0 || q[i] > vol) inside = false;
            if (inside) {
                const double rv = __drcp_rn(vol);
#pragma unroll
                for (int i = 0; i < 4; i++) lc[i] = __dmul_rn(q[i], rv);
                return 1;
            }
#pragma unroll
            for (int i = 0; i < 4; i++) lc[i] = __ddiv_rn(q[i], vol);
        } else {
            bool inside = true;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                lc[i] = __ddiv_rn(q[i], vol);
                if (lc[i] < 0 || lc[i] > 1.0) inside = false;
            }
            if (inside) return 1;
        }
        int min_i = 0;
        double min_lc = lc[0];
#pragma unroll
        for (int i = 1; i < 4; i++)
            if (lc[i] < min_lc) {
                min_lc = lc[i];
                min_i = i;
            }
        int nb = __ldg(&t->cell_con[min_i]);
        if (nb < 0) {
            if (exit_face) *exit_face = min_i;  // the face opposite vertex min_i of `cell`
            return 0;
        }
        if (hops >= limit) return -1;
        cell = nb;
        hops++;
    }
}

}  // namespace mp
