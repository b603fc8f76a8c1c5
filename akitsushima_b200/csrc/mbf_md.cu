// Velocity-Verlet NVE on the device: the two half kicks, the drift with the
// wrap into the cell, and a fixed-order kinetic-energy sum, split around the
// force call so a whole rebuild interval can be captured in one CUDA graph.
// The first half kick also carries the step's list-validity check, the
// second the kinetic-energy sum (completion counters: the block that
// finishes last does the per-step serial work), so a step is the force
// call plus two launches.
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

// md_kick_drift fused with the list-validity check of the same step: each
// atom's minimum-image displacement from the reference positions (the
// lattice is fixed, engine/neighborlist.py:661-668), its per-structure
// maximum (warp max, then one atomic per warp; max is order-free), and in
// the block that finishes last the reference's rebuild decision
// r_list - 2 d <= r_cut (:653-673): d logged, the gate word and the graph
// conditional set, the maxima and the completion word reset to 0.
__global__ void md_kick_drift_check(SysView S, double *__restrict__ pos, double *__restrict__ vel,
                                    const double *__restrict__ F, const double *__restrict__ im, double dt,
                                    const double *__restrict__ ref, unsigned long long *__restrict__ dmax,
                                    unsigned *__restrict__ done, double r_list, double r_cut,
                                    double *__restrict__ d_log, int rows, int *__restrict__ counter,
                                    int *__restrict__ gate, unsigned long long cond) {
    __shared__ bool last;
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = a < S.n_atoms;
    int s = 0;
    unsigned long long bits = 0ull;
    if (valid) {
        size_t o = 3 * (size_t)a;
        double h = 0.5 * dt * im[a];
        double vx = vel[o] + h * F[o], vy = vel[o + 1] + h * F[o + 1], vz = vel[o + 2] + h * F[o + 2];
        double x = pos[o] + dt * vx, y = pos[o + 1] + dt * vy, z = pos[o + 2] + dt * vz;
        s = S.n_struct > 1 ? S.atom_struct[a] : 0;
        const double *c = S.cells + 18 * (size_t)s;
        double s0 = x * c[9] + y * c[12] + z * c[15];
        double s1 = x * c[10] + y * c[13] + z * c[16];
        double s2 = x * c[11] + y * c[14] + z * c[17];
        s0 -= floor(s0);
        s1 -= floor(s1);
        s2 -= floor(s2);
        if (s0 >= 1.0) s0 = 0.0;
        if (s1 >= 1.0) s1 = 0.0;
        if (s2 >= 1.0) s2 = 0.0;
        double px = s0 * c[0] + s1 * c[3] + s2 * c[6];
        double py = s0 * c[1] + s1 * c[4] + s2 * c[7];
        double pz = s0 * c[2] + s1 * c[5] + s2 * c[8];
        pos[o] = px;
        pos[o + 1] = py;
        pos[o + 2] = pz;
        vel[o] = vx;
        vel[o + 1] = vy;
        vel[o + 2] = vz;
        double dx, dy, dz;
        mic_exact(c, px - ref[o], py - ref[o + 1], pz - ref[o + 2], dx, dy, dz);
        bits = (unsigned long long)__double_as_longlong(sqrt(dx * dx + dy * dy + dz * dz));
    }
    int s_first = __shfl_sync(MBF_FULL, s, 0);
    if (__all_sync(MBF_FULL, s == s_first || !valid)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long b = __shfl_xor_sync(MBF_FULL, bits, o);
            bits = b > bits ? b : bits;
        }
        if ((threadIdx.x & 31) == 0 && bits) atomicMax(dmax + s_first, bits);
    } else if (valid) {
        atomicMax(dmax + s, bits);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    int row = *counter % rows;
    int need = 0;
    for (int q = 0; q < S.n_struct; ++q) {
        double d = __longlong_as_double((long long)atomicExch(dmax + q, 0ull));
        d_log[(size_t)row * S.n_struct + q] = d;
        if (r_list - 2.0 * d <= r_cut) need = 1;
    }
    *gate = need;
    if (cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, need ? 1u : 0u);
    *counter += 1;
    *done = 0u;
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
// The block that finishes last then sums the partials into the thermo row
// (md_thermo's arithmetic, so the same bits) and resets `done`.
__device__ void md_thermo_body(int n_struct, int P, const double *__restrict__ partial,
                               const double *__restrict__ energy, double *__restrict__ thermo, int rows,
                               int *__restrict__ counter, double *sh);

__global__ void __launch_bounds__(MD_BLOCK) md_kick(SysView S, double *__restrict__ vel,
                                                    const double *__restrict__ F,
                                                    const double *__restrict__ im, double dt, int P,
                                                    double *__restrict__ partial,
                                                    const double *__restrict__ energy,
                                                    double *__restrict__ thermo, int rows,
                                                    int *__restrict__ counter, unsigned *__restrict__ done) {
    __shared__ double sh[MD_BLOCK / 32];
    __shared__ bool last;
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
    if (threadIdx.x == 0) {
        partial[(size_t)s * P + blockIdx.x] = acc;
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x * gridDim.y - 1;
    }
    __syncthreads();
    if (!last) return;
    md_thermo_body(S.n_struct, P, partial, energy, thermo, rows, counter, sh);
    if (threadIdx.x == 0) *done = 0u;
}

// The second half kick of one step and the first half kick, drift and
// list-validity check of the next, in one launch (the two kicks use the same
// forces): per atom md_kick's arithmetic, its kinetic-energy term from the
// mid-step velocity, then md_kick_drift_check's arithmetic on that velocity,
// so every stored value has the bits of the two separate launches.  Grid and
// partial sums as md_kick (blocks of one structure, blockIdx.y = s, so the
// displacement maximum of a warp belongs to one structure); the block that
// finishes last writes the thermo row of the step that ended and then takes
// the rebuild decision of the next (md_kick_drift_check's tail).
__global__ void __launch_bounds__(MD_BLOCK) md_kick_kick_drift_check(
    SysView S, double *__restrict__ pos, double *__restrict__ vel, const double *__restrict__ F,
    const double *__restrict__ im, double dt, int P, double *__restrict__ partial,
    const double *__restrict__ energy, double *__restrict__ thermo, int rows, int *__restrict__ tcounter,
    const double *__restrict__ ref, unsigned long long *__restrict__ dmax, double r_list, double r_cut,
    double *__restrict__ d_log, int *__restrict__ scounter, int *__restrict__ gate, unsigned long long cond,
    unsigned *__restrict__ done) {
    __shared__ double sh[MD_BLOCK / 32];
    __shared__ bool last;
    int s = blockIdx.y;
    int beg = S.n_struct > 1 ? S.struct_off[s] : 0;
    int end = S.n_struct > 1 ? S.struct_off[s + 1] : S.n_atoms;
    const double *c = S.cells + 18 * (size_t)s;
    double acc = 0.0;
    unsigned long long bits = 0ull;
    int first = beg + blockIdx.x * MD_CHUNK;
#pragma unroll
    for (int k = 0; k < MD_ITEMS; ++k) {
        int a = first + k * MD_BLOCK + threadIdx.x;
        if (a < end) {
            size_t o = 3 * (size_t)a;
            double w = im[a];
            double h = 0.5 * dt * w;
            double fx = F[o], fy = F[o + 1], fz = F[o + 2];
            double vx = vel[o] + h * fx, vy = vel[o + 1] + h * fy, vz = vel[o + 2] + h * fz;
            acc += (vx * vx + vy * vy + vz * vz) / w;
            vx = vx + h * fx;
            vy = vy + h * fy;
            vz = vz + h * fz;
            double x = pos[o] + dt * vx, y = pos[o + 1] + dt * vy, z = pos[o + 2] + dt * vz;
            double s0 = x * c[9] + y * c[12] + z * c[15];
            double s1 = x * c[10] + y * c[13] + z * c[16];
            double s2 = x * c[11] + y * c[14] + z * c[17];
            s0 -= floor(s0);
            s1 -= floor(s1);
            s2 -= floor(s2);
            if (s0 >= 1.0) s0 = 0.0;
            if (s1 >= 1.0) s1 = 0.0;
            if (s2 >= 1.0) s2 = 0.0;
            double px = s0 * c[0] + s1 * c[3] + s2 * c[6];
            double py = s0 * c[1] + s1 * c[4] + s2 * c[7];
            double pz = s0 * c[2] + s1 * c[5] + s2 * c[8];
            pos[o] = px;
            pos[o + 1] = py;
            pos[o + 2] = pz;
            vel[o] = vx;
            vel[o + 1] = vy;
            vel[o + 2] = vz;
            double dx, dy, dz;
            mic_exact(c, px - ref[o], py - ref[o + 1], pz - ref[o + 2], dx, dy, dz);
            unsigned long long b = (unsigned long long)__double_as_longlong(sqrt(dx * dx + dy * dy + dz * dz));
            bits = b > bits ? b : bits;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long b = __shfl_xor_sync(MBF_FULL, bits, o);
        bits = b > bits ? b : bits;
    }
    if ((threadIdx.x & 31) == 0 && bits) atomicMax(dmax + s, bits);
    acc = block_sum<MD_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partial[(size_t)s * P + blockIdx.x] = acc;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (!last) return;
    md_thermo_body(S.n_struct, P, partial, energy, thermo, rows, tcounter, sh);
    if (threadIdx.x != 0) return;
    int row = *scounter % rows;
    int need = 0;
    for (int q = 0; q < S.n_struct; ++q) {
        double d = __longlong_as_double((long long)atomicExch(dmax + q, 0ull));
        d_log[(size_t)row * S.n_struct + q] = d;
        if (r_list - 2.0 * d <= r_cut) need = 1;
    }
    *gate = need;
    if (cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, need ? 1u : 0u);
    *scounter += 1;
    *done = 0u;
}

// With inv_mass = conv / m the partials hold sum m v^2 / conv, so the
// kinetic energy is half their sum, in eV (the reference's
// 0.5 sum m v^2 / EV_ANG_TO_AMU_ANG_FS2, :243-244).
__device__ void md_thermo_body(int n_struct, int P, const double *__restrict__ partial,
                               const double *__restrict__ energy, double *__restrict__ thermo, int rows,
                               int *__restrict__ counter, double *sh) {
    int row = *counter % rows;
    for (int s = 0; s < n_struct; ++s) {
        double v = 0.0;
        for (int k = threadIdx.x; k < P; k += MD_BLOCK) v += __ldcg(partial + (size_t)s * P + k);
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
                int *counter, unsigned *done, void *stream) {
    if (!sys || !velocities || !forces || !inv_mass || !energy || !partial || !thermo || !counter || !done ||
        thermo_rows <= 0 || sys->n_struct <= 0 || sys->n_struct > 65535)
        return MBF_ERR_ARGUMENT;
    SysView S = make_view(sys);
    cudaStream_t st = (cudaStream_t)stream;
    int P = mbf_md_partial_count(sys->n_atoms);
    PROF_BEGIN("md_kick", st);
    md_kick<<<dim3(P, sys->n_struct), MD_BLOCK, 0, st>>>(S, velocities, forces, inv_mass, dt, P, partial, energy,
                                                         thermo, thermo_rows, counter, done);
    PROF_END("md_kick", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_md_kick_drift_check(const mbf_system *sys, double *positions, double *velocities, const double *forces,
                            const double *inv_mass, double dt, const double *ref_positions, double r_list,
                            double r_cut, unsigned long long *d_max, unsigned *done, double *d_log, int rows,
                            int *counter, int *gate, unsigned long long cond_handle, void *stream) {
    if (!sys || !positions || !velocities || !forces || !inv_mass || positions != sys->positions ||
        !ref_positions || !d_max || !done || !d_log || !counter || !gate || rows <= 0 || !(r_list > r_cut) ||
        !(r_cut > 0.0) || sys->n_struct <= 0 || sys->n_atoms <= 0)
        return MBF_ERR_ARGUMENT;
    SysView S = make_view(sys);
    cudaStream_t st = (cudaStream_t)stream;
    PROF_BEGIN("md_kick_drift", st);
    md_kick_drift_check<<<(sys->n_atoms + MD_BLOCK - 1) / MD_BLOCK, MD_BLOCK, 0, st>>>(
        S, positions, velocities, forces, inv_mass, dt, ref_positions, d_max, done, r_list, r_cut, d_log, rows,
        counter, gate, cond_handle);
    PROF_END("md_kick_drift", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_md_kick_kick_drift_check(const mbf_system *sys, double *positions, double *velocities,
                                 const double *forces, const double *inv_mass, double dt, const double *energy,
                                 double *partial, double *thermo, int thermo_rows, int *thermo_counter,
                                 const double *ref_positions, double r_list, double r_cut,
                                 unsigned long long *d_max, double *d_log, int rows, int *skin_counter, int *gate,
                                 unsigned long long cond_handle, unsigned *done, void *stream) {
    if (!sys || !positions || !velocities || !forces || !inv_mass || positions != sys->positions || !energy ||
        !partial || !thermo || thermo_rows <= 0 || !thermo_counter || !ref_positions || !d_max || !d_log ||
        rows <= 0 || !skin_counter || !gate || !done || !(r_list > r_cut) || !(r_cut > 0.0) ||
        sys->n_struct <= 0 || sys->n_struct > 65535 || sys->n_atoms <= 0)
        return MBF_ERR_ARGUMENT;
    SysView S = make_view(sys);
    cudaStream_t st = (cudaStream_t)stream;
    int P = mbf_md_partial_count(sys->n_atoms);
    PROF_BEGIN("md_kick_kick_drift", st);
    md_kick_kick_drift_check<<<dim3(P, sys->n_struct), MD_BLOCK, 0, st>>>(
        S, positions, velocities, forces, inv_mass, dt, P, partial, energy, thermo, thermo_rows, thermo_counter,
        ref_positions, d_max, r_list, r_cut, d_log, skin_counter, gate, cond_handle, done);
    PROF_END("md_kick_kick_drift", st);
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
