/* mini_pic_cuda.h -- drop-in replacement for the device side of the
 * reference's src/mini-pic.cpp, in the reference's own C++ types.
 *
 * A maintainer compiles mini_pic_cuda.cpp next to the reference's sources
 * (src/{maths,FESolver,meshes,particles,parameters,trace}.cpp), removes the
 * SYCL DeviceData and MoveParticles from src/mini-pic.cpp, and links
 * libminipic_cuda.so.  main() keeps calling
 *     DeviceData device(volume);
 *     MoveParticles(ions, volume, solver, params, device);
 * unchanged, and may route the field solve to the device as well:
 *     computePhiDevice(solver, ions.den, params.fesolver_method, device);
 *     updateEfDevice(solver, device);
 * Errors print a message and exit(-1), as the reference does. */
#ifndef MINI_PIC_CUDA_H
#define MINI_PIC_CUDA_H

#include <cstddef>
#include <vector>

#include "FESolver.h"
#include "meshes.h"
#include "parameters.h"
#include "particles.h"
#include "minipic_cuda.h"

/* Replaces the SYCL DeviceData of src/mini-pic.cpp:39-53, 322-355: owns one
 * mp_ctx (CUDA stream + device buffers), uploads the mesh once. */
struct DeviceData {
    mp_ctx *ctx = nullptr;
    int n_nodes = 0;
    int n_elements = 0;
    bool fe_ready = false;
    int form = MP_FORM_FP64;  /* MP_FORM_MIXED: FP32 particles and TF32 factorization */
    /* MP_FE_STORAGE_SPARSE (set before the first computePhiDevice): K is kept
     * sparse only, and computePhiDevice maps Lapack to MP_METHOD_SPARSE_CG and
     * NonLinear to MP_METHOD_SPARSE_NEWTON (Gauss-Seidel is not available). */
    int fe_storage = MP_FE_STORAGE_DENSE;
    DeviceData(Volume &volume);
    ~DeviceData();
    DeviceData(const DeviceData &) = delete;
    DeviceData &operator=(const DeviceData &) = delete;
    void reserveParticles(size_t n);
};

/* src/mini-pic.cpp:268-320: the host particle vector is copied to the device,
 * pushed (E gather, kick, drift, XtoLtet walk, density scatter), and the
 * survivors come back in the reference's order with the normalised density in
 * ions.den. */
void MoveParticles(Species &ions, Volume &volume, FESolver &solver, const Parameters &params, DeviceData &device);

/* FESolver::computePhi (src/FESolver.cpp:604-619) on the device: d and uh are
 * written back into solver.d and solver.uh.  The first call uploads K, F0, ID,
 * NX, detJ and g from the solver (after preAssembly). */
void computePhiDevice(FESolver &solver, double *ion_den, FESolver::Method method, DeviceData &device);

/* FESolver::updateEf (src/FESolver.cpp:622-636) on the device from solver.uh;
 * the field is written back into solver.ef. */
void updateEfDevice(FESolver &solver, DeviceData &device);

/* LoadVolumeMesh's geometry (src/meshes.cpp:87-262) computed on the device for
 * a Volume whose nodes (positions) and elements (con) are filled: the
 * orientation fix, volumes, alpha..delta, cell_con, node volumes and the OPEN
 * node types, written into the reference's records bit for bit as its own
 * loader computes them.  A maintainer calls it where LoadVolumeMesh's
 * geometry loops are. */
void MeshGeometryDevice(Volume &volume);

/* LoadSurfaceMesh's inlet part (src/meshes.cpp:300-353) on the device for the
 * volume.inlet_faces whose con are filled: the owning tet, u, v, the unit
 * normal and the area.  Exits like the reference when a face is held by no tet
 * or by two. */
void InletFacesDevice(Volume &volume, bool invert_normals);

/* OutputMesh (src/meshes.cpp:358-447) from the device's potential, field and
 * density (those of the last computePhiDevice, updateEfDevice and
 * MoveParticles), byte for byte the reference's file; asynchronous (the file
 * is complete after the next output call, OutputWaitDevice or ~DeviceData). */
void OutputMeshDevice(int ts, Volume &volume, DeviceData &device);
/* OutputParticles (src/particles.cpp:21-45): particles.vtp from the device's
 * particles (those MoveParticles left), asynchronous like OutputMeshDevice. */
void OutputParticlesDevice(DeviceData &device);
void OutputWaitDevice(DeviceData &device);

#endif
