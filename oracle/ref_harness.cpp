/* Test infrastructure: a C-callable harness around the reference's own compiled
 * translation units (src/{maths,FESolver,meshes,particles,parameters,trace}.cpp,
 * built unchanged from their location by oracle/Makefile into oracle/_ref/).
 *
 * It is a checker only.  Nothing in the product links or calls it; the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * The reference's driver file src/mini-pic.cpp cannot be compiled here (it needs
 * <sycl/sycl.hpp>), so the three pieces of it that the hot path uses are restated
 * below, each citing the lines it follows:
 *   - InjectIons            src/mini-pic.cpp:208-265
 *   - the SYCL kernel body  src/mini-pic.cpp:287-308 (calls the reference's own
 *                           inline XtoLtet from src/meshes.h:75-100)
 *   - MoveParticles' host   src/mini-pic.cpp:268-320 (erase_if + normalisation)
 * Everything else (mesh geometry, FESolver, LAPACK call, RNG) is the reference's
 * compiled code.  Calls into FESolver's NonLinear method may exit(-1) on
 * non-convergence exactly like the reference; tests run those in a subprocess.
 */
#include <algorithm>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>
#include <random>
#include <unistd.h>

#include "FESolver.h"
#include "maths.h"
#include "meshes.h"
#include "parameters.h"
#include "particles.h"
#include "trace.h"
#ifdef REF_WITH_SHIM
#include "mini_pic_cuda.h"
#endif

/* The reference's RNG state, a global of src/maths.cpp:17 with external linkage. */
extern std::mt19937 mt_gen;

/* The reference defines these two globals in src/mini-pic.cpp:31-32. */
int trace::enabled = 0;
Trace trace::current = Trace("__TRACE_BASE__");

namespace {

struct RefSim {
    Parameters params;
    Volume volume;
    FESolver *solver = nullptr;
    Species *ions = nullptr;
    explicit RefSim(const std::string &f) : params(f) {}
    ~RefSim() {
        delete ions;
        delete solver;
    }
};

std::string join(const std::string &dir, const std::string &f) {
    if (dir.empty() || (!f.empty() && f[0] == '/')) return f;
    return dir + "/" + f;
}

/* src/mini-pic.cpp:287-308, one particle. */
inline void push_one(Particle &part, const Tetra *elements, const double (*ef)[3], double *den,
                     double q_over_m, double dt, bool atomic) {
    for (int i = 0; i < 3; i++) part.vel[i] += q_over_m * ef[part.cell_index][i] * dt;
    for (int i = 0; i < 3; i++) part.pos[i] += part.vel[i] * dt;
    if (XtoLtet(part, elements)) {
        const Tetra &tet = elements[part.cell_index];
        for (int v = 0; v < 4; v++) {
            if (atomic) {
#pragma omp atomic
                den[tet.con[v]] += part.lc[v];
            } else {
                den[tet.con[v]] += part.lc[v];
            }
        }
    } else {
        part.cell_index = -1;
    }
}

}  // namespace

extern "C" {

int ref_sizeof_tetra() { return (int)sizeof(Tetra); }
int ref_sizeof_particle() { return (int)sizeof(Particle); }
int ref_sizeof_node() { return (int)sizeof(Node); }

/* Parameters + LoadVolumeMesh + inlet/wall LoadSurfaceMesh (src/mini-pic.cpp:75-82),
 * with the deck's mesh file names taken relative to deck_dir. */
void *ref_open(const char *deck_dir) {
    std::string dir(deck_dir);
    RefSim *s = new RefSim(join(dir, "system.param"));
    for (auto &kv : s->params.mesh_files) kv.second = join(dir, kv.second);
    if (!LoadVolumeMesh(s->params.mesh_files["global_mesh"], s->volume) ||
        !LoadSurfaceMesh(s->params.mesh_files["inlet_mesh"], s->volume, INLET, s->params.invert_normals) ||
        !LoadSurfaceMesh(s->params.mesh_files["wall_mesh"], s->volume, FIXED, s->params.invert_normals)) {
        delete s;
        return nullptr;
    }
    return s;
}

/* An extra Dirichlet surface (the sphere of the inclusion decks). */
int ref_add_fixed_surface(void *h, const char *path) {
    RefSim *s = (RefSim *)h;
    return LoadSurfaceMesh(path, s->volume, FIXED, s->params.invert_normals) ? 0 : -1;
}

/* FESolver ctor and the reference values of src/mini-pic.cpp:87-102. */
void ref_init_solver(void *h) {
    RefSim *s = (RefSim *)h;
    s->solver = new FESolver(s->volume);
    s->solver->phi0 = 0;
    s->solver->n0 = s->params.plasma_den;
    s->solver->kTe = Kb * s->params.electron_temperature;
    int n_nodes = (int)s->volume.nodes.size();
    for (int n = 0; n < n_nodes; n++) {
        if (s->volume.nodes[n].type == INLET) s->solver->g[n] = 0;
        else if (s->volume.nodes[n].type == FIXED) s->solver->g[n] = -s->params.wall_potential;
        else s->solver->g[n] = 0;
    }
}

void ref_set_g(void *h, int node, double value) { ((RefSim *)h)->solver->g[node] = value; }

/* src/mini-pic.cpp:107-108 */
void ref_assemble(void *h) {
    RefSim *s = (RefSim *)h;
    s->solver->startAssembly();
    s->solver->preAssembly();
}

/* Species + the overrides of src/mini-pic.cpp:113-116 (mass in AMU). */
void ref_init_species(void *h, double spwt, double mass_amu) {
    RefSim *s = (RefSim *)h;
    s->ions = new Species((int)s->volume.nodes.size(), s->params.plasma_species);
    s->ions->charge = 1 * QE;
    s->ions->mass = mass_amu * AMU;
    s->ions->spwt = spwt;
    for (size_t n = 0; n < s->volume.nodes.size(); n++) s->ions->den[n] = 0;
}

void ref_close(void *h) { delete (RefSim *)h; }

int ref_n_nodes(void *h) { return (int)((RefSim *)h)->volume.nodes.size(); }
int ref_n_tets(void *h) { return (int)((RefSim *)h)->volume.elements.size(); }
int ref_n_inlet(void *h) { return (int)((RefSim *)h)->volume.inlet_faces.size(); }
int ref_neq(void *h) { return ((RefSim *)h)->solver->neq; }
long ref_n_particles(void *h) { return (long)((RefSim *)h)->ions->particles.size(); }
double ref_rem(void *h) { return ((RefSim *)h)->ions->rem; }

/* double params: 0 plasma_den 1 ion_velocity 2 electron_temperature 3 wall_potential
 * 4 dt 5 kTe 6 n0 7 phi0 8 charge 9 mass 10 spwt; int 11 max_iter 12 method 13 species */
double ref_param(void *h, int which) {
    RefSim *s = (RefSim *)h;
    switch (which) {
        case 0: return s->params.plasma_den;
        case 1: return s->params.ion_velocity;
        case 2: return s->params.electron_temperature;
        case 3: return s->params.wall_potential;
        case 4: return s->params.dt;
        case 5: return s->solver ? s->solver->kTe : 0;
        case 6: return s->solver ? s->solver->n0 : 0;
        case 7: return s->solver ? s->solver->phi0 : 0;
        case 8: return s->ions ? s->ions->charge : 0;
        case 9: return s->ions ? s->ions->mass : 0;
        case 10: return s->ions ? s->ions->spwt : 0;
        case 11: return s->params.max_iter;
        case 12: return (double)s->params.fesolver_method;
        case 13: return (double)s->params.plasma_species;
    }
    return 0;
}

void ref_get_tetra_raw(void *h, void *out) {
    RefSim *s = (RefSim *)h;
    std::memcpy(out, s->volume.elements.data(), s->volume.elements.size() * sizeof(Tetra));
}

void ref_get_nodes(void *h, double *pos, int *type, double *volume) {
    RefSim *s = (RefSim *)h;
    for (size_t n = 0; n < s->volume.nodes.size(); n++) {
        const Node &nd = s->volume.nodes[n];
        for (int d = 0; d < 3; d++) pos[3 * n + d] = nd.pos[d];
        type[n] = (int)nd.type;
        volume[n] = nd.volume;
    }
}

void ref_get_inlet(void *h, int *con, double *area, double *u, double *v, int *cell_con, double *normal) {
    RefSim *s = (RefSim *)h;
    for (size_t f = 0; f < s->volume.inlet_faces.size(); f++) {
        const Face &fc = s->volume.inlet_faces[f];
        for (int i = 0; i < 3; i++) {
            con[3 * f + i] = fc.con[i];
            u[3 * f + i] = fc.u[i];
            v[3 * f + i] = fc.v[i];
            normal[3 * f + i] = fc.normal[i];
        }
        area[f] = fc.area;
        cell_con[f] = fc.cell_con;
    }
}

void ref_get_fe(void *h, int *ID, int *LM, double *NX, double *detJ) {
    RefSim *s = (RefSim *)h;
    FESolver &S = *s->solver;
    int nn = (int)s->volume.nodes.size(), ne = (int)s->volume.elements.size();
    for (int n = 0; n < nn; n++) ID[n] = S.ID[n];
    for (int e = 0; e < ne; e++) {
        detJ[e] = S.detJ[e];
        for (int a = 0; a < 4; a++) {
            LM[4 * e + a] = S.LM[e][a];
            for (int d = 0; d < 3; d++) NX[12 * e + 3 * a + d] = S.NX[e][a][d];
        }
    }
}

/* which: 0 K, 1 J (full neq x neq, row-major) */
void ref_get_matrix(void *h, int which, double *out) {
    FESolver &S = *((RefSim *)h)->solver;
    double **M = which == 0 ? S.K : S.J;
    for (int i = 0; i < S.neq; i++) std::memcpy(out + (size_t)i * S.neq, M[i], sizeof(double) * S.neq);
}

/* vectors: 0 F0[neq] 1 F1[neq] 2 d[neq] 3 g[nodes] 4 uh[nodes] 5 den[nodes] 6 ef[tets*3] */
static double *vec_ptr(RefSim *s, int which, size_t *len) {
    FESolver *S = s->solver;
    size_t nn = s->volume.nodes.size(), ne = s->volume.elements.size();
    switch (which) {
        case 0: *len = S->neq; return S->F0;
        case 1: *len = S->neq; return S->F1;
        case 2: *len = S->neq; return S->d;
        case 3: *len = nn; return S->g;
        case 4: *len = nn; return S->uh;
        case 5: *len = nn; return s->ions->den;
        case 6: *len = 3 * ne; return &S->ef[0][0];
    }
    *len = 0;
    return nullptr;
}
void ref_get_vec(void *h, int which, double *out) {
    size_t n;
    double *p = vec_ptr((RefSim *)h, which, &n);
    if (p) std::memcpy(out, p, n * sizeof(double));
}
void ref_set_vec(void *h, int which, const double *in) {
    size_t n;
    double *p = vec_ptr((RefSim *)h, which, &n);
    if (p) std::memcpy(p, in, n * sizeof(double));
}

void ref_get_particles(void *h, void *out) {
    RefSim *s = (RefSim *)h;
    std::memcpy(out, s->ions->particles.data(), s->ions->particles.size() * sizeof(Particle));
}
void ref_set_particles(void *h, const void *in, long n) {
    RefSim *s = (RefSim *)h;
    s->ions->particles.resize(n);
    std::memcpy(s->ions->particles.data(), in, n * sizeof(Particle));
}
void ref_set_rem(void *h, double rem) { ((RefSim *)h)->ions->rem = rem; }

/* InjectIons, src/mini-pic.cpp:208-265 (uses the reference's rnd() and evalEf). */
int ref_inject(void *h) {
    RefSim *s = (RefSim *)h;
    Species &ions = *s->ions;
    Volume &volume = s->volume;
    FESolver &solver = *s->solver;
    Parameters &params = s->params;
    int total_new_particles = 0;
    for (auto face : volume.inlet_faces) {
        double num_per_sec = params.plasma_den * params.ion_velocity * face.area;
        double num_real = num_per_sec * params.dt;
        double fnum_mp = num_real / ions.spwt + ions.rem;
        int num_mp = (int)fnum_mp;
        ions.rem = fnum_mp - num_mp;
        for (int p = 0; p < num_mp; p++) {
            Particle part;
            double a = rnd();
            double b = rnd();
            if ((a + b) > 1) {
                a = 1 - a;
                b = 1 - b;
            }
            for (int i = 0; i < 3; i++) {
                part.pos[i] = a * face.u[i] + b * face.v[i] + volume.nodes[face.con[0]].pos[i];
                part.vel[i] = face.normal[i] * params.ion_velocity;
            }
            part.cell_index = face.cell_con;
            double ef_part[3];
            solver.evalEf(ef_part, part.cell_index);
            for (int i = 0; i < 3; i++) part.vel[i] -= ions.charge / ions.mass * ef_part[i] * (0.5 * params.dt);
            ions.particles.push_back(part);
        }
        total_new_particles += num_mp;
    }
    return total_new_particles;
}

/* The device half of MoveParticles (src/mini-pic.cpp:275-308) without the host
 * compaction: den is zeroed and accumulated, exits get cell_index=-1.
 * nthreads<=1 runs the particles in order; otherwise an OpenMP parallel-for with
 * atomic adds, the way a SYCL CPU backend runs the parallel_for. */
void ref_push_only(void *h, int nthreads) {
    RefSim *s = (RefSim *)h;
    Species &ions = *s->ions;
    int n_nodes = (int)s->volume.nodes.size();
    for (int n = 0; n < n_nodes; n++) ions.den[n] = 0.0;
    Particle *particles = ions.particles.data();
    const Tetra *elements = s->volume.elements.data();
    const double(*ef)[3] = s->solver->ef;
    double *den = ions.den;
    double q_over_m = ions.charge / ions.mass;
    double dt = s->params.dt;
    long n_parts = (long)ions.particles.size();
    if (nthreads <= 1) {
        for (long p = 0; p < n_parts; p++) push_one(particles[p], elements, ef, den, q_over_m, dt, false);
    } else {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long p = 0; p < n_parts; p++) push_one(particles[p], elements, ef, den, q_over_m, dt, true);
    }
}

/* MoveParticles' host epilogue, src/mini-pic.cpp:316-319. Returns removed count. */
long ref_compact_normalise(void *h) {
    RefSim *s = (RefSim *)h;
    Species &ions = *s->ions;
    size_t before = ions.particles.size();
    std::erase_if(ions.particles, [](const Particle &part) { return part.cell_index < 0; });
    int n_nodes = (int)s->volume.nodes.size();
    for (int n = 0; n < n_nodes; n++) ions.den[n] *= ions.spwt / s->volume.nodes[n].volume;
    return (long)(before - ions.particles.size());
}

/* Whole MoveParticles (src/mini-pic.cpp:268-320). */
long ref_move(void *h, int nthreads) {
    ref_push_only(h, nthreads);
    return ref_compact_normalise(h);
}

/* FESolver pieces, each the reference's own method. */
void ref_compute_phi(void *h, int method) {
    RefSim *s = (RefSim *)h;
    s->solver->computePhi(s->ions->den, (FESolver::Method)method);
}
void ref_update_ef(void *h) { ((RefSim *)h)->solver->updateEf(); }
void ref_build_f1(void *h, const double *ion_den) { ((RefSim *)h)->solver->buildF1Vector((double *)ion_den); }
void ref_build_j(void *h, int method) { ((RefSim *)h)->solver->buildJmatrix((FESolver::Method)method); }
/* G = K d - F0 - F1 with the reference's matVecMultiply/vecVecSubtract (FESolver.cpp:333-335). */
void ref_residual(void *h, double *G) {
    FESolver &S = *((RefSim *)h)->solver;
    matVecMultiply(G, S.K, S.d, S.neq);
    vecVecSubtract(G, G, S.F0, S.neq);
    vecVecSubtract(G, G, S.F1, S.neq);
}
/* x is in/out (the reference's solve() passes a zeroed y). */
void ref_solve_gs(void *h, const double *b, double *x) {
    FESolver &S = *((RefSim *)h)->solver;
    S.solveLinear(S.J, x, (double *)b);
}
void ref_solve_lapack(void *h, const double *b, double *x) {
    FESolver &S = *((RefSim *)h)->solver;
    S.solveLinearLapack(S.J, x, (double *)b);
}

/* Bounded CPU timing of MoveParticles over `steps` steps on the current
 * population (no injection): returns particle-steps/s; *seconds gets the time. */
double ref_time_move(void *h, int steps, int nthreads, double *seconds) {
    RefSim *s = (RefSim *)h;
    double psteps = 0;
    auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < steps; k++) {
        psteps += (double)s->ions->particles.size();
        ref_move(h, nthreads);
    }
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    if (seconds) *seconds = sec;
    return sec > 0 ? psteps / sec : 0;
}

int ref_max_threads() { return omp_get_max_threads(); }

/* Restarts the reference's RNG stream (the process-wide mt19937 of maths.cpp),
 * so every simulation opened in one process injects like a fresh `mini-pic`. */
void ref_reseed(unsigned seed) { mt_gen.seed(seed); }

/* The reference's OutputMesh (src/meshes.cpp:358-447) and OutputParticles
 * (src/particles.cpp:21-45) write into the current directory; these run them
 * with `dir` as the current directory and return the seconds they took. */
double ref_output_mesh(void *h, int ts, const char *dir) {
    RefSim &S = *(RefSim *)h;
    char here[4096];
    if (!getcwd(here, sizeof here) || chdir(dir) != 0) return -1;
    auto t0 = std::chrono::steady_clock::now();
    OutputMesh(ts, S.volume, S.solver->uh, S.solver->ef, S.ions->den);
    auto t1 = std::chrono::steady_clock::now();
    if (chdir(here) != 0) return -1;
    return std::chrono::duration<double>(t1 - t0).count();
}
double ref_output_particles(void *h, const char *dir) {
    RefSim &S = *(RefSim *)h;
    char here[4096];
    if (!getcwd(here, sizeof here) || chdir(dir) != 0) return -1;
    auto t0 = std::chrono::steady_clock::now();
    OutputParticles(S.ions->particles);
    auto t1 = std::chrono::steady_clock::now();
    if (chdir(here) != 0) return -1;
    return std::chrono::duration<double>(t1 - t0).count();
}


#ifdef REF_WITH_SHIM
/* The device path through the C++ drop-in (mini-fem-pic-main_b200/shim): the
 * same Species, Volume, FESolver and Parameters objects, handed to the
 * reference's own signatures as main() would hand them. */
void *ref_shim_device(void *h) { return new DeviceData(((RefSim *)h)->volume); }
void ref_shim_free(void *d) { delete (DeviceData *)d; }
void ref_shim_move(void *h, void *d) {
    RefSim *s = (RefSim *)h;
    MoveParticles(*s->ions, s->volume, *s->solver, s->params, *(DeviceData *)d);
}
void ref_shim_compute_phi(void *h, void *d, int method) {
    RefSim *s = (RefSim *)h;
    computePhiDevice(*s->solver, s->ions->den, (FESolver::Method)method, *(DeviceData *)d);
}
void ref_shim_update_ef(void *h, void *d) { updateEfDevice(*((RefSim *)h)->solver, *(DeviceData *)d); }

/* The drop-in's MeshGeometryDevice + InletFacesDevice on a copy of the loaded
 * Volume whose geometry is cleared and whose tets carry the mesh file's vertex
 * order (con_file, 0-based: the reference's loader computes each volume in that
 * order before it flips the orientation); returns how many values differ from
 * what the reference's own loaders computed (0 = bit for bit).  Node types are
 * compared as OPEN or not, for the nodes the surface loads did not retype. */
long ref_shim_mesh_check(void *h, const int *con_file) {
    RefSim &S = *(RefSim *)h;
    Volume v;
    v.nodes = S.volume.nodes;
    v.elements = S.volume.elements;
    v.inlet_faces = S.volume.inlet_faces;
    for (size_t e = 0; e < v.elements.size(); e++)
        for (int k = 0; k < 4; k++) v.elements[e].con[k] = con_file[4 * e + k];
    for (Tetra &t : v.elements) {
        t.volume = 0;
        for (int k = 0; k < 4; k++) t.alpha[k] = t.beta[k] = t.gamma[k] = t.delta[k] = 0, t.cell_con[k] = -7;
    }
    for (Node &n : v.nodes) {
        n.volume = 0;
        if (n.type == OPEN) n.type = NORMAL;
    }
    for (Face &f : v.inlet_faces) {
        f.area = 0;
        f.cell_con = -7;
        for (int k = 0; k < 3; k++) f.u[k] = f.v[k] = f.normal[k] = 0;
    }
    MeshGeometryDevice(v);
    InletFacesDevice(v, S.params.invert_normals);
    long cnt[12] = {};
    for (size_t e = 0; e < v.elements.size(); e++) {
        const Tetra &a = v.elements[e], &b = S.volume.elements[e];
        cnt[0] += std::memcmp(&a.volume, &b.volume, sizeof(double)) != 0;
        cnt[1] += std::memcmp(a.con, b.con, sizeof a.con) != 0;
        cnt[2] += std::memcmp(a.alpha, b.alpha, sizeof a.alpha) != 0;
        cnt[3] += std::memcmp(a.beta, b.beta, sizeof a.beta) != 0;
        cnt[4] += std::memcmp(a.gamma, b.gamma, sizeof a.gamma) != 0;
        cnt[5] += std::memcmp(a.delta, b.delta, sizeof a.delta) != 0;
        cnt[6] += std::memcmp(a.cell_con, b.cell_con, sizeof a.cell_con) != 0;
    }
    for (size_t n = 0; n < v.nodes.size(); n++) {
        const Node &a = v.nodes[n], &b = S.volume.nodes[n];
        cnt[7] += std::memcmp(&a.volume, &b.volume, sizeof(double)) != 0;
        if (b.type == NORMAL || b.type == OPEN) cnt[8] += (a.type == OPEN) != (b.type == OPEN);
    }
    for (size_t f = 0; f < v.inlet_faces.size(); f++) {
        const Face &a = v.inlet_faces[f], &b = S.volume.inlet_faces[f];
        cnt[9] += a.cell_con != b.cell_con;
        cnt[10] += std::memcmp(&a.area, &b.area, sizeof(double)) != 0;
        cnt[11] += std::memcmp(a.u, b.u, sizeof a.u) != 0 || std::memcmp(a.v, b.v, sizeof a.v) != 0 ||
                   std::memcmp(a.normal, b.normal, sizeof a.normal) != 0;
    }
    long bad = 0;
    for (long c : cnt) bad += c;
    if (bad) {
        static const char *names[12] = {"volume", "con", "alpha", "beta", "gamma", "delta", "cell_con",
                                        "node_volume", "open", "inlet_cell", "inlet_area", "inlet_u_v_normal"};
        for (int i = 0; i < 12; i++)
            if (cnt[i]) fprintf(stderr, "mesh check: %s differs in %ld records\n", names[i], cnt[i]);
    }
    return bad;
}

void ref_shim_set_storage(void *d, int storage) { ((DeviceData *)d)->fe_storage = storage; }

/* OutputMeshDevice + OutputParticlesDevice with `dir` as the current directory. */
int ref_shim_output(void *h, void *d, int ts, const char *dir) {
    RefSim &S = *(RefSim *)h;
    char here[4096];
    if (!getcwd(here, sizeof here) || chdir(dir) != 0) return -1;
    OutputMeshDevice(ts, S.volume, *(DeviceData *)d);
    OutputParticlesDevice(*(DeviceData *)d);
    OutputWaitDevice(*(DeviceData *)d);
    return chdir(here) == 0 ? 0 : -1;
}
#endif

}  /* extern "C" */
