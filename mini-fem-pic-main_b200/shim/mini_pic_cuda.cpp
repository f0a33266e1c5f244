// Drop-in replacement for the device side of src/mini-pic.cpp over the C ABI
// of libminipic_cuda.so (declarations and usage in mini_pic_cuda.h).
#include "mini_pic_cuda.h"

#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <vector>

namespace {

// The reference reports fatal errors on std::cerr and calls exit(-1).
void check(int rc, const mp_ctx *ctx, const char *what) {
    if (rc == MP_OK) return;
    const char *msg = ctx ? mp_last_error(ctx) : nullptr;
    std::cerr << "mini-pic (CUDA): " << what << " failed: " << mp_error_string(rc);
    if (msg && *msg) std::cerr << " (" << msg << ")";
    std::cerr << std::endl;
    exit(-1);
}

void setup_fe(FESolver &solver, DeviceData &device) {
    if (device.fe_ready) return;
    // NX[e][a][d] (double***) packed to [n_tets][4][3]
    std::vector<double> nx(12 * (size_t)device.n_elements);
    for (int e = 0; e < device.n_elements; e++)
        for (int a = 0; a < 4; a++)
            for (int d = 0; d < 3; d++) nx[12 * (size_t)e + 3 * a + d] = solver.NX[e][a][d];
    mp_fe_desc fe{};
    fe.neq = solver.neq;
    fe.ID = solver.ID;
    fe.nx = nx.data();
    fe.detJ = solver.detJ;
    fe.g = solver.g;
    fe.K_rows = solver.K;
    fe.K_dense = nullptr;
    fe.F0 = solver.F0;
    fe.n0 = solver.n0;
    fe.phi0 = solver.phi0;
    fe.kTe = solver.kTe;
    check(mp_set_fe_storage(device.ctx, device.fe_storage), device.ctx, "FE storage");
    check(mp_fe_setup(device.ctx, &fe), device.ctx, "FE setup");
    device.fe_ready = true;
}

}  // namespace

DeviceData::DeviceData(Volume &volume) {
    n_nodes = (int)volume.nodes.size();
    n_elements = (int)volume.elements.size();
    if (n_nodes == 0 || n_elements == 0) check(MP_ERR_ARG, nullptr, "DeviceData (empty mesh)");
    const Tetra &t0 = volume.elements[0];
    const Node &n0 = volume.nodes[0];
    const int64_t ts = sizeof(Tetra), ns = sizeof(Node);
    mp_mesh_desc m{};
    m.n_nodes = n_nodes;
    m.n_tets = n_elements;
    m.con = t0.con;           m.con_stride = ts;
    m.volume = &t0.volume;    m.volume_stride = ts;
    m.alpha = t0.alpha;       m.alpha_stride = ts;
    m.beta = t0.beta;         m.beta_stride = ts;
    m.gamma = t0.gamma;       m.gamma_stride = ts;
    m.delta = t0.delta;       m.delta_stride = ts;
    m.cell_con = t0.cell_con; m.cell_con_stride = ts;
    m.node_pos = n0.pos;      m.node_pos_stride = ns;
    m.node_volume = &n0.volume; m.node_volume_stride = ns;
    check(mp_create(0, &m, &ctx), nullptr, "DeviceData (mp_create)");
}

DeviceData::~DeviceData() { mp_destroy(ctx); }

void DeviceData::reserveParticles(size_t n) { check(mp_particles_reserve(ctx, (int64_t)n), ctx, "reserveParticles"); }

void MoveParticles(Species &ions, Volume &volume, FESolver &solver, const Parameters &params, DeviceData &device) {
    (void)volume;
    mp_ctx *ctx = device.ctx;
    const size_t n = ions.particles.size();
    // the field of the last solve, as the reference copies solver.ef every step
    check(mp_fe_upload(ctx, MP_VEC_EF, &solver.ef[0][0]), ctx, "E field upload");
    check(mp_particles_clear(ctx), ctx, "particle clear");
    if (device.form != MP_FORM_FP64) check(mp_set_particle_form(ctx, MP_FORM_FP64), ctx, "particle form");
    if (n) {
        device.reserveParticles(n);
        Particle &p0 = ions.particles[0];
        const int64_t ps = sizeof(Particle);
        // InjectIons already applied the half-step rewind on the host
        check(mp_particles_append(ctx, (int64_t)n, p0.pos, ps, p0.vel, ps, &p0.cell_index, ps, 0, 0.0, 0.0), ctx,
              "particle upload");
    }
    if (device.form != MP_FORM_FP64) check(mp_set_particle_form(ctx, device.form), ctx, "particle form");
    mp_step_stats st{};
    check(mp_push_scatter(ctx, ions.charge / ions.mass, params.dt, ions.spwt, ions.den, &st), ctx, "MoveParticles");
    ions.particles.resize((size_t)st.n_after);
    if (st.n_after) {
        Particle &p0 = ions.particles[0];
        const int64_t ps = sizeof(Particle);
        // injection order: the order std::erase_if leaves in the reference
        check(mp_particles_download(ctx, st.n_after, p0.pos, ps, p0.vel, ps, &p0.cell_index, ps, p0.lc, ps, nullptr,
                                    MP_ORDER_ID),
              ctx, "particle download");
    }
}

void computePhiDevice(FESolver &solver, double *ion_den, FESolver::Method method, DeviceData &device) {
    setup_fe(solver, device);
    mp_newton_stats st{};
    int m = (int)method;
    if (device.fe_storage == MP_FE_STORAGE_SPARSE)
        m = method == FESolver::NonLinear ? MP_METHOD_SPARSE_NEWTON
            : method == FESolver::Lapack  ? MP_METHOD_SPARSE_CG
                                          : m;  // Gauss-Seidel needs the dense J: reported as an error
    const int rc = mp_compute_phi(device.ctx, ion_den, m, device.form, &st);
    // src/FESolver.cpp:600: each Gauss-Seidel solve that ran out of sweeps warns, the step goes on
    for (int k = 0; k < st.linear_failures; k++)
        std::cerr << " GS failed to converge in " << st.linear_iterations << " iterations, " << std::setprecision(3)
                  << ": L2=" << st.linear_residual << std::endl;
    if (rc == MP_ERR_NOT_CONVERGED) {
        // src/FESolver.cpp:360-361
        std::cerr << "NR failed to converge, L2 = " << st.l2 << std::endl;
        exit(-1);
    }
    check(rc, device.ctx, "computePhi");
    check(mp_field_download(device.ctx, solver.d, solver.uh, nullptr), device.ctx, "field download");
}

void updateEfDevice(FESolver &solver, DeviceData &device) {
    setup_fe(solver, device);
    check(mp_update_ef(device.ctx, solver.uh), device.ctx, "updateEf");
    check(mp_field_download(device.ctx, nullptr, nullptr, &solver.ef[0][0]), device.ctx, "field download");
}

void MeshGeometryDevice(Volume &volume) {
    const int nn = (int)volume.nodes.size(), nt = (int)volume.elements.size();
    std::vector<double> pos(3 * (size_t)nn), vol(nt), al(4 * (size_t)nt), be(4 * (size_t)nt), ga(4 * (size_t)nt),
        de(4 * (size_t)nt), nvol(nn);
    std::vector<int32_t> con(4 * (size_t)nt), cc(4 * (size_t)nt), open(nn);
    for (int n = 0; n < nn; n++)
        for (int d = 0; d < 3; d++) pos[3 * (size_t)n + d] = volume.nodes[n].pos[d];
    for (int e = 0; e < nt; e++)
        for (int v = 0; v < 4; v++) con[4 * (size_t)e + v] = volume.elements[e].con[v];
    check(mp_mesh_geometry_device(0, nn, pos.data(), nt, con.data(), vol.data(), al.data(), be.data(), ga.data(),
                                  de.data(), cc.data(), nvol.data(), open.data()),
          nullptr, "mesh geometry");
    for (int e = 0; e < nt; e++) {
        Tetra &t = volume.elements[e];
        t.volume = vol[e];
        for (int v = 0; v < 4; v++) {
            const size_t k = 4 * (size_t)e + v;
            t.con[v] = con[k];
            t.alpha[v] = al[k];
            t.beta[v] = be[k];
            t.gamma[v] = ga[k];
            t.delta[v] = de[k];
            t.cell_con[v] = cc[k];
        }
    }
    for (int n = 0; n < nn; n++) {
        volume.nodes[n].volume = nvol[n];
        if (open[n]) volume.nodes[n].type = OPEN;
    }
}

void InletFacesDevice(Volume &volume, bool invert_normals) {
    const int nn = (int)volume.nodes.size(), nt = (int)volume.elements.size();
    const int nf = (int)volume.inlet_faces.size();
    std::vector<double> pos(3 * (size_t)nn), u(3 * (size_t)nf), v(3 * (size_t)nf), nrm(3 * (size_t)nf), area(nf);
    std::vector<int32_t> con(4 * (size_t)nt), fc(3 * (size_t)nf), cell(nf);
    for (int n = 0; n < nn; n++)
        for (int d = 0; d < 3; d++) pos[3 * (size_t)n + d] = volume.nodes[n].pos[d];
    for (int e = 0; e < nt; e++)
        for (int k = 0; k < 4; k++) con[4 * (size_t)e + k] = volume.elements[e].con[k];
    for (int f = 0; f < nf; f++)
        for (int k = 0; k < 3; k++) fc[3 * (size_t)f + k] = volume.inlet_faces[f].con[k];
    const int rc = mp_inlet_faces_device(0, nn, pos.data(), nt, con.data(), nf, fc.data(), invert_normals ? 1 : 0,
                                         cell.data(), u.data(), v.data(), nrm.data(), area.data());
    if (rc == MP_ERR_ARG) {
        // src/meshes.cpp:318-326
        std::cerr << "Inlet surface attached to no volume element or to more than one" << std::endl;
        exit(-1);
    }
    check(rc, nullptr, "inlet faces");
    for (int f = 0; f < nf; f++) {
        Face &F = volume.inlet_faces[f];
        F.cell_con = cell[f];
        F.area = area[f];
        for (int k = 0; k < 3; k++) {
            F.u[k] = u[3 * (size_t)f + k];
            F.v[k] = v[3 * (size_t)f + k];
            F.normal[k] = nrm[3 * (size_t)f + k];
        }
    }
}

void OutputMeshDevice(int ts, Volume &volume, DeviceData &device) {
    static_assert(sizeof(NodeType) == sizeof(int32_t), "NodeType is read as int32");
    check(mp_output_mesh(device.ctx, ts, nullptr, reinterpret_cast<const int32_t *>(&volume.nodes[0].type),
                         (int64_t)sizeof(Node)),
          device.ctx, "OutputMesh");
}

void OutputParticlesDevice(DeviceData &device) {
    check(mp_output_particles(device.ctx, "particles.vtp"), device.ctx, "OutputParticles");
}

void OutputWaitDevice(DeviceData &device) { check(mp_output_wait(device.ctx), device.ctx, "output"); }
