// Mesh setup on the device.  The same outputs, bit for bit, as the host
// helpers mp_mesh_geometry, mp_inlet_faces and mp_fe_geometry:
//   - LoadVolumeMesh's geometry (src/meshes.cpp:87-262): orientation fix and
//     volumes, the barycentric coefficients alpha..delta, face neighbours,
//     node volumes, OPEN marking;
//   - LoadSurfaceMesh's inlet faces (src/meshes.cpp:290-353): owning tet,
//     u, v, unit normal, area;
//   - FESolver's ID, NX and detJ (src/FESolver.cpp:108-118, 207-287).
// Every value is the reference's expression evaluated in its order with
// separately rounded operations (__dmul_rn / __dadd_rn / __dsub_rn /
// __ddiv_rn / __dsqrt_rn), so no FMA contraction changes a bit.
//
// Face adjacency.  The reference finds a tet's neighbours by scanning the tets
// around its nodes and an inlet face's tet by scanning every tet.  Here the
// 4 faces of every tet are keyed by their sorted node triple and sorted (two
// stable radix passes: the third node, then the first two), so the two tets of
// an interior face are neighbours in the sorted list and an inlet face is a
// binary search: O(tets log tets) work, all of it on the device.  Node volumes
// are summed per node over its (tet, corner) list in tet order (a stable sort
// by node), which is the reference's accumulation order.
#include <algorithm>
#include <cstring>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "mp_internal.h"

namespace mp {
namespace {

constexpr int TH = 256;

__device__ __forceinline__ double det3(double a00, double a01, double a02, double a10, double a11, double a12,
                                       double a20, double a21, double a22) {
    // src/maths.cpp det3: M00*(M11*M22-M12*M21) - M01*(M10*M22-M12*M20) + M02*(M10*M21-M11*M20)
    const double t0 = __dmul_rn(a00, __dsub_rn(__dmul_rn(a11, a22), __dmul_rn(a12, a21)));
    const double t1 = __dmul_rn(a01, __dsub_rn(__dmul_rn(a10, a22), __dmul_rn(a12, a20)));
    const double t2 = __dmul_rn(a02, __dsub_rn(__dmul_rn(a10, a21), __dmul_rn(a11, a20)));
    return __dadd_rn(__dsub_rn(t0, t1), t2);
}

// Volumes and orientation (src/meshes.cpp:87-108): V = det4([1 x y z] rows)/6,
// nodes 1 and 3 swapped where V < 0.
__global__ void k_tet_volume(int n_tets, const double *__restrict__ pos, int *con, double *volume) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_tets) return;
    int c[4];
    for (int v = 0; v < 4; v++) c[v] = con[4 * l + v];
    double M[4][4];
    for (int v = 0; v < 4; v++) {
        M[v][0] = 1;
        for (int d = 0; d < 3; d++) M[v][d + 1] = pos[3ll * c[v] + d];
    }
    // det4 by cofactors of row 0 (src/maths.cpp), minors of rows 1..3
    const double d0 = det3(M[1][1], M[1][2], M[1][3], M[2][1], M[2][2], M[2][3], M[3][1], M[3][2], M[3][3]);
    const double d1 = det3(M[1][0], M[1][2], M[1][3], M[2][0], M[2][2], M[2][3], M[3][0], M[3][2], M[3][3]);
    const double d2 = det3(M[1][0], M[1][1], M[1][3], M[2][0], M[2][1], M[2][3], M[3][0], M[3][1], M[3][3]);
    const double d3 = det3(M[1][0], M[1][1], M[1][2], M[2][0], M[2][1], M[2][2], M[3][0], M[3][1], M[3][2]);
    const double det = __dsub_rn(__dadd_rn(__dsub_rn(__dmul_rn(M[0][0], d0), __dmul_rn(M[0][1], d1)),
                                           __dmul_rn(M[0][2], d2)),
                                 __dmul_rn(M[0][3], d3));
    double vol = __dmul_rn(1.0 / 6.0, det);
    if (vol < 0) {
        con[4 * l + 1] = c[3];
        con[4 * l + 3] = c[1];
        vol = -vol;
    }
    volume[l] = vol;
}

// Barycentric coefficients (src/meshes.cpp:111-176), [n_tets][4] each.
__global__ void k_tet_coeffs(int n_tets, const double *__restrict__ pos, const int *__restrict__ con, double *alpha,
                             double *beta, double *gamma, double *delta) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_tets) return;
    const int perm[4][3] = {{1, 2, 3}, {3, 2, 0}, {3, 0, 1}, {1, 0, 2}};
    for (int v = 0; v < 4; v++) {
        const double *p2 = pos + 3ll * con[4 * l + perm[v][0]];
        const double *p3 = pos + 3ll * con[4 * l + perm[v][1]];
        const double *p4 = pos + 3ll * con[4 * l + perm[v][2]];
        alpha[4 * l + v] = det3(p2[0], p2[1], p2[2], p3[0], p3[1], p3[2], p4[0], p4[1], p4[2]);
        beta[4 * l + v] = det3(1, p2[1], p2[2], 1, p3[1], p3[2], 1, p4[1], p4[2]);
        gamma[4 * l + v] = det3(1, p2[0], p2[2], 1, p3[0], p3[2], 1, p4[0], p4[2]);
        delta[4 * l + v] = det3(1, p2[0], p2[1], 1, p3[0], p3[1], 1, p4[0], p4[1]);
    }
}

__device__ __forceinline__ void sort3(int &a, int &b, int &c) {
    if (a > b) { int t = a; a = b; b = t; }
    if (b > c) { int t = b; b = c; c = t; }
    if (a > b) { int t = a; a = b; b = t; }
}

// Face f = 4 l + v is the face opposite vertex v of tet l.
__global__ void k_face_keys(int n_tets, const int *__restrict__ con, unsigned long long *ab, unsigned *c3, int *idx) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= 4 * n_tets) return;
    const int l = f >> 2, v = f & 3;
    int a = con[4 * l + ((v + 1) & 3)], b = con[4 * l + ((v + 2) & 3)], c = con[4 * l + ((v + 3) & 3)];
    sort3(a, b, c);
    ab[f] = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
    c3[f] = (unsigned)c;
    idx[f] = f;
}

__global__ void k_gather_ab(int m, const unsigned long long *__restrict__ ab, const int *__restrict__ idx,
                            unsigned long long *out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) out[j] = ab[idx[j]];
}

__global__ void k_gather_c(int m, const unsigned *__restrict__ c3, const int *__restrict__ idx, unsigned *out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) out[j] = c3[idx[j]];
}

// Neighbours: in the sorted face list equal keys are adjacent; a key held by
// three faces is not a valid mesh.
__global__ void k_face_pairs(int m, const unsigned long long *__restrict__ ab, const unsigned *__restrict__ c3,
                             const int *__restrict__ idx, int *cell_con, unsigned *bad) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const bool eq_prev = j > 0 && ab[j - 1] == ab[j] && c3[j - 1] == c3[j];
    const bool eq_next = j + 1 < m && ab[j + 1] == ab[j] && c3[j + 1] == c3[j];
    if (eq_prev && eq_next) atomicOr(bad, 1u);
    cell_con[idx[j]] = eq_prev ? idx[j - 1] >> 2 : eq_next ? idx[j + 1] >> 2 : -1;
}

// One tet corner's node-volume term (src/meshes.cpp:231-251): the centroid's
// lc[v] (XtoLtet's (1/6)(alpha - x beta + y gamma - z delta)/V) times V.
__global__ void k_corner_volume(int n_tets, const double *__restrict__ pos, const int *__restrict__ con,
                                const double *__restrict__ alpha, const double *__restrict__ beta,
                                const double *__restrict__ gamma, const double *__restrict__ delta,
                                const double *__restrict__ volume, double *term, unsigned *node_key, int *corner) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_tets) return;
    double x[3];
    for (int d = 0; d < 3; d++) {
        x[d] = 0;
        for (int v = 0; v < 4; v++) x[d] = __dadd_rn(x[d], __dmul_rn(0.25, pos[3ll * con[4 * l + v] + d]));
    }
    const double V = volume[l];
    for (int v = 0; v < 4; v++) {
        const int k = 4 * l + v;
        const double s = __dadd_rn(__dsub_rn(alpha[k], __dmul_rn(x[0], beta[k])), __dmul_rn(x[1], gamma[k]));
        const double lc = __ddiv_rn(__dmul_rn(1.0 / 6.0, __dsub_rn(s, __dmul_rn(x[2], delta[k]))), V);
        term[k] = __dmul_rn(lc, V);
        node_key[k] = (unsigned)con[k];
        corner[k] = k;
    }
}

// Node n's volume: its corner terms summed from zero in tet order.
__global__ void k_node_volume(int m, const unsigned *__restrict__ key, const int *__restrict__ corner,
                              const double *__restrict__ term, double *node_volume) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m || (j > 0 && key[j - 1] == key[j])) return;  // the first corner of each node's run
    double s = 0;
    for (int t = j; t < m && key[t] == key[j]; t++) s = __dadd_rn(s, term[corner[t]]);
    node_volume[key[j]] = s;
}

// OPEN marking (src/meshes.cpp:254-262).
__global__ void k_mark_open(int n_tets, const int *__restrict__ con, const int *__restrict__ cell_con, int *open) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_tets) return;
    for (int v = 0; v < 4; v++)
        if (cell_con[4 * l + v] < 0)
            for (int i = 0; i < 4; i++)
                if (i != v) open[con[4 * l + i]] = 1;
}

// Inlet faces (src/meshes.cpp:300-353): the owning tet by binary search over
// the sorted face keys (exactly one tet must hold the face), then u, v, the
// unit normal and the area in the reference's arithmetic.
__global__ void k_inlet(int n_faces, const int *__restrict__ face_con, const double *__restrict__ pos, int m,
                        const unsigned long long *__restrict__ ab, const unsigned *__restrict__ c3,
                        const int *__restrict__ idx, int invert, int *cell, double *u, double *v, double *normal,
                        double *area, unsigned *bad) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const int n1 = face_con[3 * f], n2 = face_con[3 * f + 1], n3 = face_con[3 * f + 2];
    int a = n1, b = n2, c = n3;
    sort3(a, b, c);
    const unsigned long long kab = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
    const unsigned kc = (unsigned)c;
    int lo = 0, hi = m;  // first position with key >= (kab, kc)
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const bool less = ab[mid] < kab || (ab[mid] == kab && c3[mid] < kc);
        if (less) lo = mid + 1;
        else hi = mid;
    }
    const bool found = lo < m && ab[lo] == kab && c3[lo] == kc;
    const bool twice = found && lo + 1 < m && ab[lo + 1] == kab && c3[lo + 1] == kc;
    if (!found || twice) {
        atomicOr(bad, 1u);
        cell[f] = -1;
        return;
    }
    cell[f] = idx[lo] >> 2;
    const double *p1 = pos + 3ll * n1, *p2 = pos + 3ll * n2, *p3 = pos + 3ll * n3;
    double uu[3], vv[3];
    for (int i = 0; i < 3; i++) {
        uu[i] = __dsub_rn(p2[i], p1[i]);
        vv[i] = __dsub_rn(p3[i], p1[i]);
        u[3 * f + i] = uu[i];
        v[3 * f + i] = vv[i];
    }
    double nrm[3];
    nrm[0] = __dsub_rn(__dmul_rn(uu[2], vv[1]), __dmul_rn(uu[1], vv[2]));
    nrm[1] = __dsub_rn(__dmul_rn(uu[0], vv[2]), __dmul_rn(uu[2], vv[0]));
    nrm[2] = __dsub_rn(__dmul_rn(uu[1], vv[0]), __dmul_rn(uu[0], vv[1]));
    if (invert)
        for (int i = 0; i < 3; i++) nrm[i] = -nrm[i];
    const double len =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(nrm[0], nrm[0]), __dmul_rn(nrm[1], nrm[1])), __dmul_rn(nrm[2], nrm[2])));
    for (int i = 0; i < 3; i++) normal[3 * f + i] = __ddiv_rn(nrm[i], len);
    area[f] = __ddiv_rn(len, 2.0);
}

// FESolver::computeNX and its inverse (src/FESolver.cpp:207-287).
__global__ void k_fe_nx(int n_tets, const double *__restrict__ pos, const int *__restrict__ con, double *nx,
                        double *detJ) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    const double na_xi[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, -1, -1}};
    double x[4][3];
    for (int a = 0; a < 4; a++)
        for (int d = 0; d < 3; d++) x[a][d] = pos[3ll * con[4 * e + a] + d];
    double M[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0;
            for (int a = 0; a < 4; a++) s = __dadd_rn(s, __dmul_rn(na_xi[a][j], x[a][i]));
            M[i][j] = s;
        }
    detJ[e] = det3(M[0][0], M[0][1], M[0][2], M[1][0], M[1][1], M[1][2], M[2][0], M[2][1], M[2][2]);
    const double a = M[0][0], b = M[0][1], c = M[0][2], d = M[1][0], ee = M[1][1], f = M[1][2], g = M[2][0],
                 h = M[2][1], i = M[2][2];
    double V[3][3];
    V[0][0] = __dsub_rn(__dmul_rn(ee, i), __dmul_rn(f, h));
    V[1][0] = -__dsub_rn(__dmul_rn(d, i), __dmul_rn(f, g));
    V[2][0] = __dsub_rn(__dmul_rn(d, h), __dmul_rn(ee, g));
    V[0][1] = -__dsub_rn(__dmul_rn(b, i), __dmul_rn(c, h));
    V[1][1] = __dsub_rn(__dmul_rn(a, i), __dmul_rn(c, g));
    V[2][1] = -__dsub_rn(__dmul_rn(a, h), __dmul_rn(b, g));
    V[0][2] = __dsub_rn(__dmul_rn(b, f), __dmul_rn(c, ee));
    V[1][2] = -__dsub_rn(__dmul_rn(a, f), __dmul_rn(c, d));
    V[2][2] = __dsub_rn(__dmul_rn(a, ee), __dmul_rn(b, d));
    const double det = __dadd_rn(__dadd_rn(__dmul_rn(a, V[0][0]), __dmul_rn(b, V[1][0])), __dmul_rn(c, V[2][0]));
    double vmax = 0;
    for (int r = 0; r < 3; r++)
        for (int s = 0; s < 3; s++) vmax = fabs(V[r][s]) > vmax ? fabs(V[r][s]) : vmax;
    double idet = 0;
    if (!(__ddiv_rn(fabs(vmax), fabs(det)) > 1e12)) idet = __ddiv_rn(1.0, det);
    for (int r = 0; r < 3; r++)
        for (int s = 0; s < 3; s++) V[r][s] = __dmul_rn(V[r][s], idet);
    for (int aa = 0; aa < 4; aa++)
        for (int dd = 0; dd < 3; dd++) {
            double s = 0;
            for (int k = 0; k < 3; k++) s = __dadd_rn(s, __dmul_rn(na_xi[aa][k], V[k][dd]));
            nx[12ll * e + 3 * aa + dd] = s;
        }
}

__global__ void k_unknown_flags(int n_nodes, const int *__restrict__ type, int *flag) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < n_nodes) flag[n] = (type[n] == 0 || type[n] == 1) ? 1 : 0;
}

__global__ void k_ids(int n_nodes, const int *__restrict__ flag, const int *__restrict__ scan, int *ID) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < n_nodes) ID[n] = flag[n] ? scan[n] : -1;
}

unsigned bits_for(long long v) {
    unsigned b = 1;
    while (b < 32 && (1ll << b) <= v) b++;
    return b;
}

// Device buffers of one call, freed on every return path.
struct Scratch {
    std::vector<void *> ptrs;
    ~Scratch() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T **p, size_t n) {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(1, n));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

#define MESH_CUDA(call)                              \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) return MP_ERR_CUDA;   \
    } while (0)

// The sorted face list of a mesh: keys (ab, c3) ascending, idx = 4 tet + v.
struct FaceList {
    unsigned long long *ab = nullptr;
    unsigned *c3 = nullptr;
    int *idx = nullptr;
};

int sort_faces(Scratch &S, int n_nodes, int n_tets, const int *d_con, FaceList &out, cudaStream_t st) {
    const int m = 4 * n_tets;
    unsigned long long *ab0, *ab1, *ab2;
    unsigned *c0, *c1;
    int *i0, *i1, *i2;
    MESH_CUDA(S.alloc(&ab0, m));
    MESH_CUDA(S.alloc(&ab1, m));
    MESH_CUDA(S.alloc(&ab2, m));
    MESH_CUDA(S.alloc(&c0, m));
    MESH_CUDA(S.alloc(&c1, m));
    MESH_CUDA(S.alloc(&i0, m));
    MESH_CUDA(S.alloc(&i1, m));
    MESH_CUDA(S.alloc(&i2, m));
    const int g = (m + TH - 1) / TH;
    k_face_keys<<<g, TH, 0, st>>>(n_tets, d_con, ab0, c0, i0);
    MESH_CUDA(cudaGetLastError());
    const unsigned nb = bits_for(n_nodes);
    size_t t1 = 0, t2 = 0;
    MESH_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, c0, c1, i0, i1, m, 0, nb, st));
    MESH_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, ab1, ab2, i1, i2, m, 0, 32 + nb, st));
    void *tmp;
    MESH_CUDA(S.alloc((char **)&tmp, std::max(t1, t2)));
    size_t tb = std::max(t1, t2);
    // pass 1: by the third node; pass 2 (stable): by the first two
    MESH_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, c0, c1, i0, i1, m, 0, nb, st));
    k_gather_ab<<<g, TH, 0, st>>>(m, ab0, i1, ab1);
    MESH_CUDA(cudaGetLastError());
    tb = std::max(t1, t2);
    MESH_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, ab1, ab2, i1, i2, m, 0, 32 + nb, st));
    k_gather_c<<<g, TH, 0, st>>>(m, c0, i2, c1);
    MESH_CUDA(cudaGetLastError());
    out.ab = ab2;
    out.c3 = c1;
    out.idx = i2;
    return MP_OK;
}

int set_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return MP_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return MP_ERR_ARG;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) return MP_ERR_NO_DEVICE;
    MESH_CUDA(cudaSetDevice(device));
    return MP_OK;
}

}  // namespace
}  // namespace mp

using namespace mp;

int mp_mesh_geometry_device(int device, int32_t n_nodes, const double *node_pos, int32_t n_tets, int32_t *con,
                            double *volume, double *alpha, double *beta, double *gamma, double *delta,
                            int32_t *cell_con, double *node_volume, int32_t *node_open) {
    if (n_nodes <= 0 || n_tets <= 0 || !node_pos || !con || !volume || !alpha || !beta || !gamma || !delta ||
        !cell_con || !node_volume || n_tets > (1 << 29))
        return MP_ERR_ARG;
    for (long long t = 0; t < 4ll * n_tets; t++)
        if (con[t] < 0 || con[t] >= n_nodes) return MP_ERR_ARG;
    int rc = set_device(device);
    if (rc) return rc;
    Scratch S;
    cudaStream_t st;
    MESH_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    const int m = 4 * n_tets;
    double *d_pos, *d_vol, *d_a, *d_b, *d_g, *d_d, *d_term, *d_nvol;
    int *d_con, *d_cc, *d_corner, *d_corner2, *d_open;
    unsigned *d_key, *d_key2, *d_bad;
    MESH_CUDA(S.alloc(&d_pos, 3ll * n_nodes));
    MESH_CUDA(S.alloc(&d_con, m));
    MESH_CUDA(S.alloc(&d_vol, n_tets));
    MESH_CUDA(S.alloc(&d_a, m));
    MESH_CUDA(S.alloc(&d_b, m));
    MESH_CUDA(S.alloc(&d_g, m));
    MESH_CUDA(S.alloc(&d_d, m));
    MESH_CUDA(S.alloc(&d_cc, m));
    MESH_CUDA(S.alloc(&d_term, m));
    MESH_CUDA(S.alloc(&d_key, m));
    MESH_CUDA(S.alloc(&d_key2, m));
    MESH_CUDA(S.alloc(&d_corner, m));
    MESH_CUDA(S.alloc(&d_corner2, m));
    MESH_CUDA(S.alloc(&d_nvol, n_nodes));
    MESH_CUDA(S.alloc(&d_open, n_nodes));
    MESH_CUDA(S.alloc(&d_bad, 1));
    MESH_CUDA(cudaMemcpyAsync(d_pos, node_pos, sizeof(double) * 3 * n_nodes, cudaMemcpyHostToDevice, st));
    MESH_CUDA(cudaMemcpyAsync(d_con, con, sizeof(int) * m, cudaMemcpyHostToDevice, st));
    MESH_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), st));
    MESH_CUDA(cudaMemsetAsync(d_nvol, 0, sizeof(double) * n_nodes, st));
    MESH_CUDA(cudaMemsetAsync(d_open, 0, sizeof(int) * n_nodes, st));
    const int gt = (n_tets + TH - 1) / TH, gm = (m + TH - 1) / TH;
    k_tet_volume<<<gt, TH, 0, st>>>(n_tets, d_pos, d_con, d_vol);
    k_tet_coeffs<<<gt, TH, 0, st>>>(n_tets, d_pos, d_con, d_a, d_b, d_g, d_d);
    MESH_CUDA(cudaGetLastError());
    FaceList F;
    if ((rc = sort_faces(S, n_nodes, n_tets, d_con, F, st))) return rc;
    k_face_pairs<<<gm, TH, 0, st>>>(m, F.ab, F.c3, F.idx, d_cc, d_bad);
    k_corner_volume<<<gt, TH, 0, st>>>(n_tets, d_pos, d_con, d_a, d_b, d_g, d_d, d_vol, d_term, d_key, d_corner);
    MESH_CUDA(cudaGetLastError());
    size_t tb = 0;
    const unsigned nb = bits_for(n_nodes);
    MESH_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_key, d_key2, d_corner, d_corner2, m, 0, nb, st));
    void *tmp;
    MESH_CUDA(S.alloc((char **)&tmp, tb));
    MESH_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, d_key, d_key2, d_corner, d_corner2, m, 0, nb, st));
    k_node_volume<<<gm, TH, 0, st>>>(m, d_key2, d_corner2, d_term, d_nvol);
    if (node_open) k_mark_open<<<gt, TH, 0, st>>>(n_tets, d_con, d_cc, d_open);
    MESH_CUDA(cudaGetLastError());
    unsigned bad = 0;
    MESH_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(con, d_con, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(volume, d_vol, sizeof(double) * n_tets, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(alpha, d_a, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(beta, d_b, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(gamma, d_g, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(delta, d_d, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(cell_con, d_cc, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(node_volume, d_nvol, sizeof(double) * n_nodes, cudaMemcpyDeviceToHost, st));
    if (node_open) MESH_CUDA(cudaMemcpyAsync(node_open, d_open, sizeof(int) * n_nodes, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaStreamSynchronize(st));
    return bad ? MP_ERR_ARG : MP_OK;  // a face shared by three tets
}

int mp_inlet_faces_device(int device, int32_t n_nodes, const double *node_pos, int32_t n_tets, const int32_t *con,
                          int32_t n_faces, const int32_t *face_con, int invert_normals, int32_t *cell_con, double *u,
                          double *v, double *normal, double *area) {
    if (n_nodes <= 0 || n_tets <= 0 || !node_pos || !con || n_faces < 0 || n_tets > (1 << 29) ||
        (n_faces > 0 && (!face_con || !cell_con || !u || !v || !normal || !area)))
        return MP_ERR_ARG;
    if (n_faces == 0) return MP_OK;
    for (long long t = 0; t < 4ll * n_tets; t++)
        if (con[t] < 0 || con[t] >= n_nodes) return MP_ERR_ARG;
    for (long long t = 0; t < 3ll * n_faces; t++)
        if (face_con[t] < 0 || face_con[t] >= n_nodes) return MP_ERR_ARG;
    int rc = set_device(device);
    if (rc) return rc;
    Scratch S;
    cudaStream_t st;
    MESH_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    double *d_pos, *d_u, *d_v, *d_n, *d_area;
    int *d_con, *d_fc, *d_cell;
    unsigned *d_bad;
    MESH_CUDA(S.alloc(&d_pos, 3ll * n_nodes));
    MESH_CUDA(S.alloc(&d_con, 4ll * n_tets));
    MESH_CUDA(S.alloc(&d_fc, 3ll * n_faces));
    MESH_CUDA(S.alloc(&d_cell, n_faces));
    MESH_CUDA(S.alloc(&d_u, 3ll * n_faces));
    MESH_CUDA(S.alloc(&d_v, 3ll * n_faces));
    MESH_CUDA(S.alloc(&d_n, 3ll * n_faces));
    MESH_CUDA(S.alloc(&d_area, n_faces));
    MESH_CUDA(S.alloc(&d_bad, 1));
    MESH_CUDA(cudaMemcpyAsync(d_pos, node_pos, sizeof(double) * 3 * n_nodes, cudaMemcpyHostToDevice, st));
    MESH_CUDA(cudaMemcpyAsync(d_con, con, sizeof(int) * 4 * n_tets, cudaMemcpyHostToDevice, st));
    MESH_CUDA(cudaMemcpyAsync(d_fc, face_con, sizeof(int) * 3 * n_faces, cudaMemcpyHostToDevice, st));
    MESH_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), st));
    FaceList F;
    if ((rc = sort_faces(S, n_nodes, n_tets, d_con, F, st))) return rc;
    k_inlet<<<(n_faces + TH - 1) / TH, TH, 0, st>>>(n_faces, d_fc, d_pos, 4 * n_tets, F.ab, F.c3, F.idx,
                                                     invert_normals, d_cell, d_u, d_v, d_n, d_area, d_bad);
    MESH_CUDA(cudaGetLastError());
    unsigned bad = 0;
    MESH_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(cell_con, d_cell, sizeof(int) * n_faces, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(u, d_u, sizeof(double) * 3 * n_faces, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(v, d_v, sizeof(double) * 3 * n_faces, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(normal, d_n, sizeof(double) * 3 * n_faces, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(area, d_area, sizeof(double) * n_faces, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaStreamSynchronize(st));
    return bad ? MP_ERR_ARG : MP_OK;  // 0 or more than 1 tet holding an inlet face: the reference exits
}

int mp_fe_geometry_device(int device, int32_t n_nodes, const double *node_pos, const int32_t *node_type,
                          int32_t n_tets, const int32_t *con, int32_t *ID, double *nx, double *detJ, int32_t *neq) {
    if (n_nodes <= 0 || n_tets <= 0 || !node_pos || !node_type || !con || !ID || !nx || !detJ || !neq)
        return MP_ERR_ARG;
    for (long long t = 0; t < 4ll * n_tets; t++)
        if (con[t] < 0 || con[t] >= n_nodes) return MP_ERR_ARG;
    int rc = set_device(device);
    if (rc) return rc;
    Scratch S;
    cudaStream_t st;
    MESH_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    double *d_pos, *d_nx, *d_detJ;
    int *d_con, *d_type, *d_flag, *d_scan, *d_ID;
    MESH_CUDA(S.alloc(&d_pos, 3ll * n_nodes));
    MESH_CUDA(S.alloc(&d_con, 4ll * n_tets));
    MESH_CUDA(S.alloc(&d_type, n_nodes));
    MESH_CUDA(S.alloc(&d_flag, n_nodes));
    MESH_CUDA(S.alloc(&d_scan, n_nodes));
    MESH_CUDA(S.alloc(&d_ID, n_nodes));
    MESH_CUDA(S.alloc(&d_nx, 12ll * n_tets));
    MESH_CUDA(S.alloc(&d_detJ, n_tets));
    MESH_CUDA(cudaMemcpyAsync(d_pos, node_pos, sizeof(double) * 3 * n_nodes, cudaMemcpyHostToDevice, st));
    MESH_CUDA(cudaMemcpyAsync(d_con, con, sizeof(int) * 4 * n_tets, cudaMemcpyHostToDevice, st));
    MESH_CUDA(cudaMemcpyAsync(d_type, node_type, sizeof(int) * n_nodes, cudaMemcpyHostToDevice, st));
    const int gn = (n_nodes + TH - 1) / TH;
    k_unknown_flags<<<gn, TH, 0, st>>>(n_nodes, d_type, d_flag);
    MESH_CUDA(cudaGetLastError());
    size_t tb = 0;
    MESH_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_flag, d_scan, n_nodes, st));
    void *tmp;
    MESH_CUDA(S.alloc((char **)&tmp, tb));
    MESH_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, d_flag, d_scan, n_nodes, st));
    k_ids<<<gn, TH, 0, st>>>(n_nodes, d_flag, d_scan, d_ID);
    k_fe_nx<<<(n_tets + TH - 1) / TH, TH, 0, st>>>(n_tets, d_pos, d_con, d_nx, d_detJ);
    MESH_CUDA(cudaGetLastError());
    int last_scan = 0, last_flag = 0;
    MESH_CUDA(cudaMemcpyAsync(&last_scan, d_scan + n_nodes - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(&last_flag, d_flag + n_nodes - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(ID, d_ID, sizeof(int) * n_nodes, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(nx, d_nx, sizeof(double) * 12 * n_tets, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaMemcpyAsync(detJ, d_detJ, sizeof(double) * n_tets, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaStreamSynchronize(st));
    *neq = last_scan + last_flag;
    return MP_OK;
}
