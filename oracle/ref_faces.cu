// TEST INFRASTRUCTURE (the checker, never the product): runs the
// reference's own face-drag kernel, surfaceDragForce
// (common/simulator/sim_kernel.cu:66-139), compiled from the reference's
// source, on one robot's faces in one block, so that the face law of the
// oracle (face_force_f32, mercury_oracle.c) is pinned against it.
//
// The kernel writes x + v dt + F dt^2 for every mass (F = the sum of the
// shares of its faces, accumulated with shared-memory atomics); with dt = 1
// and a large density the caller reads F back as newPos - x - v.
//
// It is launched with one warp: the kernel has no barrier between loading
// the masses into shared memory, accumulating the faces and writing back
// (sim_kernel.cu:82-131), so with several warps a warp reads corners another
// has not loaded yet, or its shares are zeroed by the owner's late load
// (measured here: whole shares lost at 256 threads).
#include "sim_kernel.cu"

#include <cstdint>
#include <vector>

extern "C" int ref_surface_drag(int n_mass, const float* pos4, const float* vel4, int n_face,
                                const uint16_t* faces3, float rho, float dt, float* new_pos4) {
    if (n_mass <= 0 || n_face <= 0 || 36 * n_mass > 48 * 1024) return -1;
    // the reference's kernel indexes its shared arrays by the corners
    // without a check: every corner must lie inside the block's masses
    std::vector<ushort4> f4((size_t)n_face);
    for (int f = 0; f < n_face; ++f) {
        const uint16_t* c = faces3 + 3 * f;
        if (c[0] >= n_mass || c[1] >= n_mass || c[2] >= n_mass) return -1;
        f4[f] = make_ushort4(c[0], c[1], c[2], 0);
    }
    SimOptions opt{};
    opt.dt = dt;
    opt.massesPerBlock = (uint)n_mass;
    opt.facesPerBlock = (uint)n_face;
    opt.boundaryMassesPerBlock = (uint)n_mass;
    opt.maxMasses = (uint)n_mass;
    opt.maxFaces = (uint)n_face;
    opt.drag = rho;
    setSimOpts(opt);
    float4 *d_pos = nullptr, *d_new = nullptr, *d_vel = nullptr;
    ushort4* d_faces = nullptr;
    const size_t mb = sizeof(float4) * (size_t)n_mass;
    cudaError_t e = cudaMalloc(&d_pos, mb);
    if (e == cudaSuccess) e = cudaMalloc(&d_new, mb);
    if (e == cudaSuccess) e = cudaMalloc(&d_vel, mb);
    if (e == cudaSuccess) e = cudaMalloc(&d_faces, sizeof(ushort4) * (size_t)n_face);
    if (e == cudaSuccess) e = cudaMemcpy(d_pos, pos4, mb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_vel, vel4, mb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_new, pos4, mb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_faces, f4.data(), sizeof(ushort4) * (size_t)n_face, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        surfaceDragForce<<<1, 32, 36 * (size_t)n_mass>>>(d_pos, d_new, d_vel, d_faces);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(new_pos4, d_new, mb, cudaMemcpyDeviceToHost);
    cudaFree(d_pos);
    cudaFree(d_new);
    cudaFree(d_vel);
    cudaFree(d_faces);
    return e == cudaSuccess ? 0 : (int)e;
}
