// Host-side setup of the hot path: the mesh geometry the kernels consume, the
// FE bookkeeping, the inlet faces and the reference injector.  All of it runs
// once per mesh (or once per step for the injector) and is arithmetic the
// reference does on the host; it is restated here with the reference's
// expression order so the device sees bit-identical inputs.  Built with
// -ffp-contract=off.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <random>
#include <unordered_map>
#include <vector>

#include "mp_injector.h"
#include "mp_internal.h"

namespace {

// det3 / det4, src/maths.cpp:22-57.
double det3(const double M[3][3]) {
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
           M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

double det4(const double M[4][4]) {
    double M0[3][3], M1[3][3], M2[3][3], M3[3][3];
    for (int i = 0; i < 3; i++) {
        M0[i][0] = M[i + 1][1]; M0[i][1] = M[i + 1][2]; M0[i][2] = M[i + 1][3];
        M1[i][0] = M[i + 1][0]; M1[i][1] = M[i + 1][2]; M1[i][2] = M[i + 1][3];
        M2[i][0] = M[i + 1][0]; M2[i][1] = M[i + 1][1]; M2[i][2] = M[i + 1][3];
        M3[i][0] = M[i + 1][0]; M3[i][1] = M[i + 1][1]; M3[i][2] = M[i + 1][2];
    }
    return M[0][0] * det3(M0) - M[0][1] * det3(M1) + M[0][2] * det3(M2) - M[0][3] * det3(M3);
}

struct FaceKey {
    int a, b, c;
    bool operator==(const FaceKey &o) const { return a == o.a && b == o.b && c == o.c; }
};
struct FaceHash {
    size_t operator()(const FaceKey &k) const {
        uint64_t h = (uint64_t)(uint32_t)k.a * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(uint32_t)k.b * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)k.c * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};
FaceKey sorted_key(int x, int y, int z) {
    int v[3] = {x, y, z};
    std::sort(v, v + 3);
    return FaceKey{v[0], v[1], v[2]};
}

}  // namespace

namespace mp {

// Quadrature points of buildF1Vector/buildJmatrix (src/FESolver.cpp:114-117,
// 497-501): l = -+sqrt(1/3), xi = 0.5*(l+1), evalNa (FESolver.cpp:188-196).
Quadrature make_quadrature() {
    Quadrature q;
    double l[2] = {-std::sqrt(1.0 / 3.0), std::sqrt(1.0 / 3.0)};
    int p = 0;
    for (int k = 0; k < 2; k++)
        for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
                double xi = 0.5 * (l[i] + 1);
                double eta = 0.5 * (l[j] + 1);
                double zeta = 0.5 * (l[k] + 1);
                q.Na[0][p] = xi;
                q.Na[1][p] = eta;
                q.Na[2][p] = zeta;
                q.Na[3][p] = 1 - xi - eta - zeta;
                p++;
            }
    return q;
}

}  // namespace mp

extern "C" {

int mp_mesh_geometry(int32_t n_nodes, const double *node_pos, int32_t n_tets, int32_t *con, double *volume,
                     double *alpha, double *beta, double *gamma, double *delta, int32_t *cell_con,
                     double *node_volume, int32_t *node_open) {
    if (n_nodes <= 0 || n_tets <= 0 || !node_pos || !con || !volume || !alpha || !beta || !gamma || !delta ||
        !cell_con || !node_volume)
        return MP_ERR_ARG;
    for (long t = 0; t < 4L * n_tets; t++)
        if (con[t] < 0 || con[t] >= n_nodes) return MP_ERR_ARG;
    auto P = [&](int n, int d) { return node_pos[3 * (long)n + d]; };
    // volumes and orientation, src/meshes.cpp:87-108
    for (int l = 0; l < n_tets; l++) {
        int *c = con + 4L * l;
        double M[4][4];
        for (int i = 0; i < 4; i++) M[i][0] = 1;
        for (int v = 0; v < 4; v++)
            for (int dim = 0; dim < 3; dim++) M[v][dim + 1] = P(c[v], dim);
        double vol = (1.0 / 6.0) * det4(M);
        if (vol < 0) {
            int t = c[1];
            c[1] = c[3];
            c[3] = t;
            vol = -vol;
        }
        volume[l] = vol;
    }
    // barycentric coefficients, src/meshes.cpp:111-176
    for (int l = 0; l < n_tets; l++) {
        const int *c = con + 4L * l;
        double M[3][3];
        for (int v = 0; v < 4; v++) {
            int v2 = 0, v3 = 0, v4 = 0;
            switch (v) {
                case 0: v2 = 1; v3 = 2; v4 = 3; break;
                case 1: v2 = 3; v3 = 2; v4 = 0; break;
                case 2: v2 = 3; v3 = 0; v4 = 1; break;
                case 3: v2 = 1; v3 = 0; v4 = 2; break;
            }
            const double *p2 = node_pos + 3L * c[v2];
            const double *p3 = node_pos + 3L * c[v3];
            const double *p4 = node_pos + 3L * c[v4];
            M[0][0] = p2[0]; M[0][1] = p2[1]; M[0][2] = p2[2];
            M[1][0] = p3[0]; M[1][1] = p3[1]; M[1][2] = p3[2];
            M[2][0] = p4[0]; M[2][1] = p4[1]; M[2][2] = p4[2];
            alpha[4L * l + v] = det3(M);
            M[0][0] = 1; M[0][1] = p2[1]; M[0][2] = p2[2];
            M[1][0] = 1; M[1][1] = p3[1]; M[1][2] = p3[2];
            M[2][0] = 1; M[2][1] = p4[1]; M[2][2] = p4[2];
            beta[4L * l + v] = det3(M);
            M[0][0] = 1; M[0][1] = p2[0]; M[0][2] = p2[2];
            M[1][0] = 1; M[1][1] = p3[0]; M[1][2] = p3[2];
            M[2][0] = 1; M[2][1] = p4[0]; M[2][2] = p4[2];
            gamma[4L * l + v] = det3(M);
            M[0][0] = 1; M[0][1] = p2[0]; M[0][2] = p2[1];
            M[1][0] = 1; M[1][1] = p3[0]; M[1][2] = p3[1];
            M[2][0] = 1; M[2][1] = p4[0]; M[2][2] = p4[1];
            delta[4L * l + v] = det3(M);
        }
    }
    // face adjacency (src/meshes.cpp:180-227): the neighbour across the face
    // opposite vertex v is the other tet holding the same three nodes.
    std::unordered_map<FaceKey, std::array<int, 2>, FaceHash> faces;
    faces.reserve((size_t)n_tets * 3);
    static const int opp[4][3] = {{1, 2, 3}, {2, 3, 0}, {3, 0, 1}, {0, 1, 2}};
    for (int l = 0; l < n_tets; l++) {
        const int *c = con + 4L * l;
        for (int v = 0; v < 4; v++) {
            FaceKey k = sorted_key(c[opp[v][0]], c[opp[v][1]], c[opp[v][2]]);
            auto it = faces.find(k);
            if (it == faces.end()) faces.emplace(k, std::array<int, 2>{l, -1});
            else if (it->second[1] < 0) it->second[1] = l;
            else return MP_ERR_ARG;  // a face shared by three tets: not a valid mesh
        }
    }
    for (int l = 0; l < n_tets; l++) {
        const int *c = con + 4L * l;
        for (int v = 0; v < 4; v++) {
            const auto &pr = faces[sorted_key(c[opp[v][0]], c[opp[v][1]], c[opp[v][2]])];
            cell_con[4L * l + v] = pr[0] == l ? pr[1] : pr[0];
        }
    }
    // node volumes from the centroid weights, src/meshes.cpp:231-251
    for (int n = 0; n < n_nodes; n++) node_volume[n] = 0;
    for (int i = 0; i < n_tets; i++) {
        const int *c = con + 4L * i;
        double pos[3];
        for (int dim = 0; dim < 3; dim++) {
            pos[dim] = 0;
            for (int v = 0; v < 4; v++) pos[dim] += 0.25 * P(c[v], dim);
        }
        for (int v = 0; v < 4; v++) {
            double lc = (1.0 / 6.0) *
                        (alpha[4L * i + v] - pos[0] * beta[4L * i + v] + pos[1] * gamma[4L * i + v] -
                         pos[2] * delta[4L * i + v]) /
                        volume[i];
            node_volume[c[v]] += lc * volume[i];
        }
    }
    // OPEN marking, src/meshes.cpp:254-262
    if (node_open) {
        for (int n = 0; n < n_nodes; n++) node_open[n] = 0;
        for (int e = 0; e < n_tets; e++)
            for (int v = 0; v < 4; v++)
                if (cell_con[4L * e + v] < 0)
                    for (int i = 0; i < 4; i++)
                        if (i != v) node_open[con[4L * e + i]] = 1;
    }
    return MP_OK;
}

int mp_fe_geometry(int32_t n_nodes, const double *node_pos, const int32_t *node_type, int32_t n_tets,
                   const int32_t *con, int32_t *ID, double *nx, double *detJ, int32_t *neq) {
    if (n_nodes <= 0 || n_tets <= 0 || !node_pos || !node_type || !con || !ID || !nx || !detJ || !neq)
        return MP_ERR_ARG;
    // ID, src/FESolver.cpp:108-112 (NORMAL=0 and OPEN=1 nodes are unknowns)
    int P = 0;
    for (int n = 0; n < n_nodes; n++) ID[n] = (node_type[n] == 0 || node_type[n] == 1) ? P++ : -1;
    *neq = P;
    // computeNX + inverse, src/FESolver.cpp:207-287
    static const double na_xi[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, -1, -1}};
    for (int e = 0; e < n_tets; e++) {
        double x[4][3];
        for (int a = 0; a < 4; a++)
            for (int d = 0; d < 3; d++) x[a][d] = node_pos[3L * con[4L * e + a] + d];
        double x_xi[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                x_xi[i][j] = 0;
                for (int a = 0; a < 4; a++) x_xi[i][j] += na_xi[a][j] * x[a][i];
            }
        detJ[e] = det3(x_xi);
        const double(&M)[3][3] = x_xi;
        double V[3][3];
        double a = M[0][0], b = M[0][1], c = M[0][2], d = M[1][0], ee = M[1][1], f = M[1][2], g = M[2][0],
               h = M[2][1], i = M[2][2];
        V[0][0] = (ee * i - f * h);
        V[1][0] = -(d * i - f * g);
        V[2][0] = (d * h - ee * g);
        V[0][1] = -(b * i - c * h);
        V[1][1] = (a * i - c * g);
        V[2][1] = -(a * h - b * g);
        V[0][2] = (b * f - c * ee);
        V[1][2] = -(a * f - c * d);
        V[2][2] = (a * ee - b * d);
        double det = a * V[0][0] + b * V[1][0] + c * V[2][0];
        double Vmax = 0;
        for (int m = 0; m < 3; m++)
            for (int n = 0; n < 3; n++) Vmax = std::fabs(V[m][n]) > Vmax ? std::fabs(V[m][n]) : Vmax;
        double idet = 0;
        if (!(std::fabs(Vmax) / std::fabs(det) > 1e12)) idet = 1 / det;
        for (int r = 0; r < 3; r++)
            for (int s = 0; s < 3; s++) V[r][s] *= idet;
        for (int aa = 0; aa < 4; aa++)
            for (int dd = 0; dd < 3; dd++) {
                double acc = 0;
                for (int k = 0; k < 3; k++) acc += na_xi[aa][k] * V[k][dd];
                nx[12L * e + 3 * aa + dd] = acc;
            }
    }
    return MP_OK;
}

int mp_inlet_faces(int32_t n_nodes, const double *node_pos, int32_t n_tets, const int32_t *con, int32_t n_faces,
                   const int32_t *face_con, int invert_normals, int32_t *cell_con, double *u, double *v,
                   double *normal, double *area) {
    if (n_faces < 0 || (n_faces > 0 && (!face_con || !cell_con || !u || !v || !normal || !area)))
        return MP_ERR_ARG;
    // the owning tet: the unique tet holding the face's three nodes (src/meshes.cpp:306-326)
    std::unordered_map<FaceKey, std::array<int, 2>, FaceHash> faces;
    static const int opp[4][3] = {{1, 2, 3}, {2, 3, 0}, {3, 0, 1}, {0, 1, 2}};
    for (int l = 0; l < n_tets; l++)
        for (int q = 0; q < 4; q++) {
            const int *c = con + 4L * l;
            FaceKey k = sorted_key(c[opp[q][0]], c[opp[q][1]], c[opp[q][2]]);
            auto it = faces.find(k);
            if (it == faces.end()) faces.emplace(k, std::array<int, 2>{l, -1});
            else it->second[1] = l;
        }
    for (int f = 0; f < n_faces; f++) {
        const int *fc = face_con + 3L * f;
        for (int i = 0; i < 3; i++)
            if (fc[i] < 0 || fc[i] >= n_nodes) return MP_ERR_ARG;
        auto it = faces.find(sorted_key(fc[0], fc[1], fc[2]));
        if (it == faces.end() || it->second[1] >= 0) return MP_ERR_ARG;  // 0 or >1 tets: reference exits
        cell_con[f] = it->second[0];
        const double *p1 = node_pos + 3L * fc[0], *p2 = node_pos + 3L * fc[1], *p3 = node_pos + 3L * fc[2];
        double *uu = u + 3L * f, *vv = v + 3L * f, *nn = normal + 3L * f;
        for (int i = 0; i < 3; i++) {
            uu[i] = p2[i] - p1[i];
            vv[i] = p3[i] - p1[i];
        }
        double nrm[3];
        nrm[0] = uu[2] * vv[1] - uu[1] * vv[2];
        nrm[1] = uu[0] * vv[2] - uu[2] * vv[0];
        nrm[2] = uu[1] * vv[0] - uu[0] * vv[1];
        if (invert_normals) {
            nrm[0] = -nrm[0];
            nrm[1] = -nrm[1];
            nrm[2] = -nrm[2];
        }
        double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        for (int i = 0; i < 3; i++) nn[i] = nrm[i] / len;
        area[f] = len / 2;
    }
    return MP_OK;
}

int mp_injector_create(int32_t n_faces, const int32_t *face_con, const double *u, const double *v,
                       const double *normal, const double *area, const int32_t *cell_con, const double *node_pos,
                       uint32_t seed, mp_injector **out) {
    if (!out || n_faces < 0 || (n_faces > 0 && (!face_con || !u || !v || !normal || !area || !cell_con || !node_pos)))
        return MP_ERR_ARG;
    mp_injector *inj = new mp_injector();
    inj->n_faces = n_faces;
    inj->con.assign(face_con, face_con + 3L * n_faces);
    inj->u.assign(u, u + 3L * n_faces);
    inj->v.assign(v, v + 3L * n_faces);
    inj->normal.assign(normal, normal + 3L * n_faces);
    inj->area.assign(area, area + n_faces);
    inj->cell.assign(cell_con, cell_con + n_faces);
    inj->p0.resize(3L * n_faces);
    for (int f = 0; f < n_faces; f++)
        for (int i = 0; i < 3; i++) inj->p0[3L * f + i] = node_pos[3L * face_con[3L * f] + i];
    inj->gen.seed(seed);
    *out = inj;
    return MP_OK;
}

int mp_injector_destroy(mp_injector *inj) {
    delete inj;
    return MP_OK;
}

int mp_injector_get_rem(mp_injector *inj, double *rem) {
    if (!inj || !rem) return MP_ERR_ARG;
    *rem = inj->rem;
    return MP_OK;
}

int mp_injector_set_rem(mp_injector *inj, double rem) {
    if (!inj) return MP_ERR_ARG;
    inj->rem = rem;
    return MP_OK;
}

int mp_injector_count(mp_injector *inj, double plasma_den, double ion_velocity, double dt, double spwt,
                      int64_t *n_next) {
    if (!inj || !n_next) return MP_ERR_ARG;
    double rem = inj->rem;
    int64_t total = 0;
    for (int f = 0; f < inj->n_faces; f++) {
        double num_per_sec = plasma_den * ion_velocity * inj->area[f];
        double num_real = num_per_sec * dt;
        double fnum_mp = num_real / spwt + rem;
        int num_mp = (int)fnum_mp;
        rem = fnum_mp - num_mp;
        total += num_mp;
    }
    *n_next = total;
    return MP_OK;
}

// InjectIons without the velocity rewind, src/mini-pic.cpp:212-262.
int mp_injector_sample(mp_injector *inj, double plasma_den, double ion_velocity, double dt, double spwt,
                       int64_t max_n, double *pos, int64_t pos_stride, double *vel, int64_t vel_stride,
                       int32_t *cell, int64_t cell_stride, int64_t *n_out) {
    if (!inj || !n_out || !pos || !vel || !cell) return MP_ERR_ARG;
    int64_t need = 0;
    int rc = mp_injector_count(inj, plasma_den, ion_velocity, dt, spwt, &need);
    if (rc != MP_OK) return rc;
    if (need > max_n) return MP_ERR_ARG;
    auto at = [](void *base, int64_t stride, int64_t i) { return (char *)base + stride * i; };
    int64_t k = 0;
    for (int f = 0; f < inj->n_faces; f++) {
        double num_per_sec = plasma_den * ion_velocity * inj->area[f];
        double num_real = num_per_sec * dt;
        double fnum_mp = num_real / spwt + inj->rem;
        int num_mp = (int)fnum_mp;
        inj->rem = fnum_mp - num_mp;
        const double *u = &inj->u[3L * f], *v = &inj->v[3L * f], *nrm = &inj->normal[3L * f], *p0 = &inj->p0[3L * f];
        for (int p = 0; p < num_mp; p++) {
            double a = inj->dist(inj->gen);
            double b = inj->dist(inj->gen);
            if ((a + b) > 1) {
                a = 1 - a;
                b = 1 - b;
            }
            double *pp = (double *)at(pos, pos_stride, k);
            double *vv = (double *)at(vel, vel_stride, k);
            for (int i = 0; i < 3; i++) {
                pp[i] = a * u[i] + b * v[i] + p0[i];
                vv[i] = nrm[i] * ion_velocity;
            }
            *(int32_t *)at(cell, cell_stride, k) = inj->cell[f];
            k++;
        }
    }
    *n_out = k;
    return MP_OK;
}

}  // extern "C"
