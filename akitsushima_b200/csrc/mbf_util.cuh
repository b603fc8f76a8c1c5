// Internal helpers shared by the kernel files (scan, reductions, layouts).
#pragma once

#include "mbf_common.cuh"

namespace mbf {

// Per-atom accumulators written by every evaluation: energy, virial[9] and
// the number of neighbours inside the cutoff.  A structure with no pair
// inside the cutoff gets energy 0, as the reference returns early then
// (engine/eam.py:237-238, engine/tersoff.py:1293-1294).
constexpr int ATOM_ACC = 11;

size_t scan_workspace_ints(int n);
// Exclusive scan of n ints into out[0..n]; out[n] is the total.  `ws` needs
// scan_workspace_ints(n) ints.
int exclusive_scan(const int *in, int *out, int n, int *ws, cudaStream_t st);

// The last step of the three-body evaluations: F_a = f_local[a] + the slot
// forces in a's row of G (n_slots x 3), with the per-structure sums of
// per_atom into energy / virial (ChunkSums below).  `sdone` (n_struct
// words, the workspace's sdone region) is cleared by the call.
int gather_reduce(int n_struct, int n_atoms, const int *row_off, const double *G, const double *f_local,
                  double *forces, const double *per_atom, const mbf_reduce_plan *plan, double *partial,
                  double *energy, double *virial, unsigned *sdone, cudaStream_t st);

// Threads per block of the fused gather kernels: 8 lanes per atom of the
// plan's mean chunk, at least 128 and at most 512.
static inline int chunk_block(int n_atoms, int n_chunks) {
    int per = n_chunks > 0 ? (n_atoms + n_chunks - 1) / n_chunks : 1;
    return per <= 16 ? 128 : (per <= 32 ? 256 : 512);
}

// The per-structure sums of the per-atom records (energy, virial, pair
// count), done by the last kernel of an evaluation: one block per chunk of
// the reduction plan (a run of atoms of one structure; 512 in the plans the
// Python Batch makes) adds its atoms' records, writes the chunk total to
// partial[c], and the block that completes a structure (a completion
// counter per structure) adds that structure's chunk totals; every sum in
// a fixed order, so the same input gives the same bits.
struct ChunkSums {
    const int *chunk;        // (n_chunks, 3): structure, first atom, end atom
    const int *chunk_first;  // (n_struct + 1,): first chunk of each structure
    const double *per_atom;  // (n_atoms, ATOM_ACC)
    double *partial;         // (n_chunks, ATOM_ACC)
    double *energy;          // (n_struct,)
    double *virial;          // (n_struct, 9)
    unsigned *sdone;         // (n_struct,) completion counters, zero at launch
};

// Block-wide end of a chunk's sums, called by every thread of an NT-thread
// block.  r0 / r1: the thread's running sums of record entries q = t % 8 and
// q = 8 + t % 8 (q < ATOM_ACC) over the atoms its 8-lane group visited.
template <int NT>
__device__ __forceinline__ void chunk_sums_finish(const ChunkSums &cs, int c, int s, double r0, double r1) {
    static_assert(NT % 32 == 0 && NT >= 64, "chunk_sums_finish: whole warps, two or more");
    constexpr int NW = NT / 32;
    constexpr int PER = NT / ATOM_ACC;   // chunk totals summed per value in the tail
    __shared__ double sh[NW][16];
    __shared__ double tail[PER * ATOM_ACC];
    __shared__ bool last;
    const int t = threadIdx.x, w = t >> 5, l = t & 31;
    r0 += __shfl_xor_sync(MBF_FULL, r0, 8);
    r1 += __shfl_xor_sync(MBF_FULL, r1, 8);
    r0 += __shfl_xor_sync(MBF_FULL, r0, 16);
    r1 += __shfl_xor_sync(MBF_FULL, r1, 16);
    if (l < 8) {
        sh[w][l] = r0;
        sh[w][8 + l] = r1;
    }
    __syncthreads();
    if (t < ATOM_ACC) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < NW; ++k) v += sh[k][t];
        cs.partial[(size_t)c * ATOM_ACC + t] = v;
        __threadfence();
    }
    __syncthreads();
    const int c0 = cs.chunk_first[s], c1 = cs.chunk_first[s + 1];
    if (t == 0) last = atomicAdd(cs.sdone + s, 1u) == (unsigned)(c1 - c0 - 1);
    __syncthreads();
    if (!last) return;
    const int q = t % ATOM_ACC, k0 = t / ATOM_ACC;
    if (k0 < PER) {
        double v = 0.0;
        for (int k = c0 + k0; k < c1; k += PER) v += __ldcg(cs.partial + (size_t)k * ATOM_ACC + q);
        tail[k0 * ATOM_ACC + q] = v;
    }
    __syncthreads();
    if (t < ATOM_ACC) {
        double v = 0.0;
        for (int k = 0; k < PER; ++k) v += tail[k * ATOM_ACC + t];
        sh[0][t] = v;
    }
    __syncthreads();
    if (t == 0) cs.energy[s] = sh[0][10] > 0.0 ? sh[0][0] : 0.0;
    if (t < 9) cs.virial[9 * (size_t)s + t] = sh[0][1 + t];
}

// Optional site-term outputs of an evaluation (all null: none): the site
// energy U_i per atom and, per list slot, dU_centre/dv and v (the
// minimum-image vector centre -> neighbour); slots outside the cutoff get
// dU/dv = 0.
struct SiteOut {
    double *e;     // (n_atoms,)
    double *dudv;  // (n_slots, 3)
    double *vec;   // (n_slots, 3)
};

// Bytes of the evaluation workspace's `err` region (the error words 0..3)
// that each evaluation clears at its start.
constexpr int ERR_CLEAR_BYTES = 16;

// Layout of the evaluation workspace (all offsets 256-byte aligned):
//   err      device error words (ints; see ERR_CLEAR_BYTES)
//   per_atom (n_atoms, ATOM_ACC) doubles
//   f_local  (n_atoms, 3) doubles (three-body potentials: centre-local force)
//   atom_aux (n_atoms, 2) doubles (EAM F'(rho), F(rho))
//   pack     (n_atoms, 4) doubles (position + F'(rho), one record per atom)
//   slot     (n_slots, 3) doubles (three-body force left on each neighbour)
//   slot_b   (n_slots, 2) doubles (Tersoff bond order and its derivative)
//   partial  (n_chunks, ATOM_ACC) doubles
//   sdone    (n_chunks,) completion counters of the per-structure sums
struct EvalLayout {
    size_t err, per_atom, f_local, atom_aux, pack, slot, slot_b, partial, sdone, total;
};

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static inline EvalLayout eval_layout(int n_atoms, long long n_slots, int n_chunks) {
    EvalLayout L;
    size_t o = 0;
    L.err = o;
    o = align256(o + 64);
    L.per_atom = o;
    o = align256(o + sizeof(double) * (size_t)n_atoms * ATOM_ACC);
    L.f_local = o;
    o = align256(o + sizeof(double) * (size_t)n_atoms * 3);
    L.atom_aux = o;
    o = align256(o + sizeof(double) * (size_t)n_atoms * 2);
    L.pack = o;
    o = align256(o + sizeof(double) * (size_t)n_atoms * 4);
    L.slot = o;
    o = align256(o + sizeof(double) * (size_t)n_slots * 3);
    L.slot_b = o;
    o = align256(o + sizeof(double) * (size_t)n_slots * 2);
    L.partial = o;
    o = align256(o + sizeof(double) * (size_t)(n_chunks > 0 ? n_chunks : 1) * ATOM_ACC);
    L.sdone = o;
    o = align256(o + sizeof(unsigned) * (size_t)(n_chunks > 0 ? n_chunks : 1));
    L.total = o;
    return L;
}

template <typename T>
static inline T *ws_at(void *ws, size_t off) {
    return reinterpret_cast<T *>(static_cast<char *>(ws) + off);
}

}  // namespace mbf

// ---- launch profiler (CUDA events on the launching stream) -----------------
// Off by default; mbf_profile_begin() turns it on.  Each PROF_LAUNCH records
// an event pair around one kernel launch; mbf_profile_end() synchronises and
// returns per-kernel counts and total milliseconds.
namespace mbf {
void prof_mark(const char *name, cudaStream_t st, bool start);
extern bool g_prof_on;
}  // namespace mbf

#define PROF_BEGIN(name, st) \
    do { if (mbf::g_prof_on) mbf::prof_mark(name, st, true); } while (0)
#define PROF_END(name, st) \
    do { if (mbf::g_prof_on) mbf::prof_mark(name, st, false); } while (0)
