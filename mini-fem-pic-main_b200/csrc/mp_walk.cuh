// The reference's barycentric coordinates and tet walk in FP64, bit for bit
// (every operation rounded on its own, in the reference's order: no FMA).
// Shared by the push kernels and the adjoint.
#pragma once

#include "mp_internal.h"

namespace mp {

constexpr double ONE_SIXTH = 1.0 / 6.0;

// Barycentric weight i of point (x,y,z) in tet t, the reference's expression
// (1.0/6.0)*(alpha - x*beta + y*gamma - z*delta)/volume in its order, unfused.
__device__ __forceinline__ void lambdas_fp64(const TetRec *__restrict__ t, double x, double y, double z,
                                             double lc[4]) {
    const double2 *a2 = reinterpret_cast<const double2 *>(t->alpha);
    const double2 *b2 = reinterpret_cast<const double2 *>(t->beta);
    const double2 *g2 = reinterpret_cast<const double2 *>(t->gamma);
    const double2 *d2 = reinterpret_cast<const double2 *>(t->delta);
    double vol = __ldg(&t->volume);
    double al[4], be[4], ga[4], de[4];
    double2 q;
    q = __ldg(a2); al[0] = q.x; al[1] = q.y; q = __ldg(a2 + 1); al[2] = q.x; al[3] = q.y;
    q = __ldg(b2); be[0] = q.x; be[1] = q.y; q = __ldg(b2 + 1); be[2] = q.x; be[3] = q.y;
    q = __ldg(g2); ga[0] = q.x; ga[1] = q.y; q = __ldg(g2 + 1); ga[2] = q.x; ga[3] = q.y;
    q = __ldg(d2); de[0] = q.x; de[1] = q.y; q = __ldg(d2 + 1); de[2] = q.x; de[3] = q.y;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        double v = __dsub_rn(al[i], __dmul_rn(x, be[i]));
        v = __dadd_rn(v, __dmul_rn(y, ga[i]));
        v = __dsub_rn(v, __dmul_rn(z, de[i]));
        v = __dmul_rn(ONE_SIXTH, v);
        lc[i] = __ddiv_rn(v, vol);
    }
}

// XtoLtet (src/meshes.h:75-100) with a hop limit.  Returns 1 inside, 0 left the
// domain, -1 hop limit reached (cell is then the last tet visited).
__device__ __forceinline__ int walk_fp64(const TetRec *__restrict__ tets, int &cell, double x, double y, double z,
                                         double lc[4], int limit, int &hops, int *exit_face = nullptr) {
    for (;;) {
        const TetRec *t = tets + cell;
        lambdas_fp64(t, x, y, z, lc);
        bool inside = true;
#pragma unroll
        for (int i = 0; i < 4; i++)
            if (lc[i] < 0 || lc[i] > 1.0) inside = false;
        if (inside) return 1;
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
