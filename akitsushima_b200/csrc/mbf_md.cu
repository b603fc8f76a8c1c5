// Velocity-Verlet NVE on the device: the two half kicks, the drift with the
// wrap into the cell, and a fixed-order kinetic-energy sum, split around the
// force call so a whole rebuild interval can be captured in one CUDA graph.
//
// Replaces the integrator of NVESimulation.run
// (solvers/molecular_dynamics.py:1969-2000) and _kinetic_energy (:239-244);
// the force call between the kicks is any of the *_eval entries.
#include <string.h>

#include "mbf_util.cuh"

namespace mbf {

constexpr int MD_BLOCK = 256;
constexpr int MD_ITEMS = 4;
constexpr int MD_CHUNK = MD_BLOCK * MD_ITEMS;

// v += dt/2 a; r += dt v; frac = r @ inv(L), frac -= floor(frac),
// frac >= 1 -> 0, r = frac @ L (the reference's wrap, :1981-1989).
__global__ void md_kick_drift(SysView S, double *__restrict__ pos, double *__restrict__ vel,
                              const double *__restrict__ F, const double *__restrict__ im, double dt) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= S.n_atoms) return;
    size_t o = 3 * (size_t)a;
    double h = 0.5 * dt * im[a];
    double vx = vel[o] + h * F[o], vy = vel[o + 1] + h * F[o + 1], vz = vel[o + 2] + h * F[o + 2];
    double x = pos[o] + dt * vx, y = pos[o + 1] + dt * vy, z = pos[o + 2] + dt * vz;
    const double *c = cell_of(S, a);
    double s0 = x * c[9] + y * c[12] + z * c[15];
    double s1 = x * c[10] + y * c[13] + z * c[16];
    double s2 = x * c[11] + y * c[14] + z * c[17];
    s0 -= floor(s0);
    s1 -= floor(s1);
    s2 -= floor(s2);
    if (s0 >= 1.0) s0 = 0.0;
    if (s1 >= 1.0) s1 = 0.0;
    if (s2 >= 1.0) s2 = 0.0;
    pos[o] = s0 * c[0] + s1 * c[3] + s2 * c[6];
    pos[o + 1] = s0 * c[1] + s1 * c[4] + s2 * c[7];
    pos[o + 2] = s0 * c[2] + s1 * c[5] + s2 * c[8];
    vel[o] = vx;
    vel[o + 1] = vy;
    vel[o + 2] = vz;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(MBF_FULL, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < NT / 32 ? sh[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(MBF_FULL, v, o);
    }
    return v;
}

// Second half kick and m v^2 over chunk blockIdx.x of structure blockIdx.y
// (mass = 1 / inv_mass in amu / conv units: conv cancels in m v^2 / conv).
__global__ void __launch_bounds__(MD_BLOCK) md_kick(SysView S, double *__restrict__ vel,
                                                    const double *__restrict__ F,
                                                    const double *__restrict__ im, double dt, int P,
                                                    double *__restrict__ partial) {
    __shared__ double sh[MD_BLOCK / 32];
    int s = blockIdx.y;
    int beg = S.n_struct > 1 ? S.struct_off[s] : 0;
    int end = S.n_struct > 1 ? S.struct_off[s + 1] : S.n_atoms;
    double acc = 0.0;
    int first = beg + blockIdx.x * MD_CHUNK;
#pragma unroll
    for (int k = 0; k < MD_ITEMS; ++k) {
        int a = first + k * MD_BLOCK + threadIdx.x;
        if (a < end) {
            size_t o = 3 * (size_t)a;
            double w = im[a];
            double h = 0.5 * dt * w;
            double vx = vel[o] + h * F[o], vy = vel[o + 1] + h * F[o + 1], vz = vel[o + 2] + h * F[o + 2];
            vel[o] = vx;
            vel[o + 1] = vy;
            vel[o + 2] = vz;
            acc += (vx * vx + vy * vy + vz * vz) / w;
        }
    }
    acc = block_sum<MD_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partial[(size_t)s * P + blockIdx.x] = acc;
}

// With inv_mass = conv / m the partials hold sum m v^2 / conv, so the
// kinetic energy is half their sum, in eV (the reference's
// 0.5 sum m v^2 / EV_ANG_TO_AMU_ANG_FS2, :243-244).
__global__ void __launch_bounds__(MD_BLOCK) md_thermo(int n_struct, int P, const double *__restrict__ partial,
                                                      const double *__restrict__ energy,
                                                      double *__restrict__ thermo, int rows,
                                                      int *__restrict__ counter) {
    __shared__ double sh[MD_BLOCK / 32];
    int row = *counter % rows;
    for (int s = 0; s < n_struct; ++s) {
        double v = 0.0;
        for (int k = threadIdx.x; k < P; k += MD_BLOCK) v += partial[(size_t)s * P + k];
        v = block_sum<MD_BLOCK>(v, sh);
        if (threadIdx.x == 0) {
            double *t = thermo + 2 * ((size_t)row * n_struct + s);
            t[0] = energy[s];
            t[1] = 0.5 * v;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter += 1;
}

}  // namespace mbf

using namespace mbf;

extern "C" {

int mbf_md_kick_drift(const mbf_system *sys, double *positions, double *velocities, const double *forces,
                      const double *inv_mass, double dt, void *stream) {
    if (!sys || !positions || !velocities || !forces || !inv_mass || positions != sys->positions)
        return MBF_ERR_ARGUMENT;
    if (sys->n_atoms == 0) return MBF_OK;
    SysView S = make_view(sys);
    cudaStream_t st = (cudaStream_t)stream;
    PROF_BEGIN("md_kick_drift", st);
    md_kick_drift<<<(sys->n_atoms + MD_BLOCK - 1) / MD_BLOCK, MD_BLOCK, 0, st>>>(S, positions, velocities, forces,
                                                                               inv_mass, dt);
    PROF_END("md_kick_drift", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_md_partial_count(int n_atoms) { return n_atoms <= 0 ? 1 : (n_atoms + MD_CHUNK - 1) / MD_CHUNK; }

int mbf_md_kick(const mbf_system *sys, double *velocities, const double *forces, const double *inv_mass,
                double dt, const double *energy, double *partial, double *thermo, int thermo_rows,
                int *counter, void *stream) {
    if (!sys || !velocities || !forces || !inv_mass || !energy || !partial || !thermo || !counter ||
        thermo_rows <= 0 || sys->n_struct <= 0 || sys->n_struct > 65535)
        return MBF_ERR_ARGUMENT;
    SysView S = make_view(sys);
    cudaStream_t st = (cudaStream_t)stream;
    int P = mbf_md_partial_count(sys->n_atoms);
    PROF_BEGIN("md_kick", st);
    md_kick<<<dim3(P, sys->n_struct), MD_BLOCK, 0, st>>>(S, velocities, forces, inv_mass, dt, P, partial);
    PROF_END("md_kick", st);
    MBF_CHECK_LAUNCH();
    md_thermo<<<1, MD_BLOCK, 0, st>>>(sys->n_struct, P, partial, energy, thermo, thermo_rows, counter);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_capture_cond_create(void *stream, unsigned long long *cond_handle) {
    if (!cond_handle) return MBF_ERR_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr) != cudaSuccess) return MBF_ERR_CUDA;
    if (cs != cudaStreamCaptureStatusActive) return MBF_ERR_ARGUMENT;
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 0u, cudaGraphCondAssignDefault) != cudaSuccess) return MBF_ERR_CUDA;
    *cond_handle = (unsigned long long)h;
    return MBF_OK;
}

int mbf_capture_if_begin(void *stream, void *body_stream, unsigned long long cond_handle) {
    cudaStream_t st = (cudaStream_t)stream, bs = (cudaStream_t)body_stream;
    if (st == bs || !cond_handle) return MBF_ERR_ARGUMENT;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps) != cudaSuccess) return MBF_ERR_CUDA;
    if (cs != cudaStreamCaptureStatusActive) return MBF_ERR_ARGUMENT;
    // the parameter union has no default constructor: zeroed storage
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams *p = reinterpret_cast<cudaGraphNodeParams *>(raw);
    p->type = cudaGraphNodeTypeConditional;
    p->conditional.handle = (cudaGraphConditionalHandle)cond_handle;
    p->conditional.type = cudaGraphCondTypeIf;
    p->conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, deps, ndeps, p) != cudaSuccess) return MBF_ERR_CUDA;
    cudaGraph_t body = p->conditional.phGraph_out[0];
    if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
        return MBF_ERR_CUDA;
    if (cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
        return MBF_ERR_CUDA;
    return MBF_OK;
}

int mbf_capture_if_end(void *body_stream) {
    cudaGraph_t g;
    if (cudaStreamEndCapture((cudaStream_t)body_stream, &g) != cudaSuccess) return MBF_ERR_CUDA;
    return MBF_OK;
}

}  // extern "C"
