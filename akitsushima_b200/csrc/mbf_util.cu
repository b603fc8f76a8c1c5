// Scan, per-structure reduction and small utilities shared by the kernels.
#include "mbf_util.cuh"

namespace mbf {

int persistent_grid(int blocks_needed, int block, const void *kernel, size_t smem) {
    static int n_sm = 0;
    if (n_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        if (n_sm <= 0) n_sm = 148;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess ||
        per_sm <= 0)
        per_sm = 1;
    int g = n_sm * per_sm;
    if (blocks_needed < g) g = blocks_needed;
    return g > 0 ? g : 1;
}

// ---- exclusive scan of int32 (n + 1 outputs: out[n] = total) -------------

constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ int warp_incl_scan(int v) {
    int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(MBF_FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ int block_excl_scan(int v, int &excl) {
    __shared__ int warp_tot[32];
    __shared__ int block_tot;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = warp_incl_scan(v);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int nw = blockDim.x >> 5;
        int t = lane < nw ? warp_tot[lane] : 0;
        int ti = warp_incl_scan(t);
        if (lane < nw) warp_tot[lane] = ti - t;
        if (lane == 31) block_tot = ti;  // nw <= 32
    }
    __syncthreads();
    excl = inc - v + warp_tot[wid];
    int total = block_tot;
    __syncthreads();
    return total;
}

__global__ void scan_tiles(const int *__restrict__ in, int *__restrict__ out, int n,
                           int *__restrict__ tile_sums) {
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int excl;
    int total = block_excl_scan(s, excl);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = excl;
        excl += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block: exclusive scan of the tile sums in place; writes the grand
// total to *total.
__global__ void scan_tile_sums(int *__restrict__ tile_sums, int n_tiles, int *__restrict__ total) {
    int carry = 0;
    for (int base = 0; base < n_tiles; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < n_tiles ? tile_sums[i] : 0;
        int excl;
        int t = block_excl_scan(v, excl);
        if (i < n_tiles) tile_sums[i] = excl + carry;
        carry += t;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_add(int *__restrict__ out, int n, const int *__restrict__ tile_sums,
                         const int *__restrict__ total) {
    int base = blockIdx.x * SCAN_TILE;
    int add = tile_sums[blockIdx.x];
    for (int k = threadIdx.x; k < SCAN_TILE; k += blockDim.x) {
        int i = base + k;
        if (i < n) out[i] += add;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = *total;
}

size_t scan_workspace_ints(int n) { return (size_t)(n + SCAN_TILE - 1) / SCAN_TILE + 2; }

int exclusive_scan(const int *in, int *out, int n, int *ws, cudaStream_t st) {
    int n_tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (n_tiles == 0) n_tiles = 1;
    int *tile_sums = ws;
    int *total = ws + n_tiles;
    scan_tiles<<<n_tiles, SCAN_BLOCK, 0, st>>>(in, out, n, tile_sums);
    scan_tile_sums<<<1, SCAN_BLOCK, 0, st>>>(tile_sums, n_tiles, total);
    scan_add<<<n_tiles, 256, 0, st>>>(out, n, tile_sums, total);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

// ---- force gather and per-structure sums -----------------------------------

// Gather the three-body forces the centres left on atom a: every centre x
// wrote the force its angles put on a into a's own slot (a -> x), so the
// row is read contiguously, 8 lanes per atom; fused with the per-structure
// sums (ChunkSums): a block per chunk of the reduction plan, each group also
// adding its atom's record (entries sub and sub + 8), the next atom's row
// bounds loaded one iteration ahead.
template <int NT>
__global__ void __launch_bounds__(NT) gather_reduce_rows(const int *__restrict__ row_off,
                                                         const double *__restrict__ G,
                                                         const double *__restrict__ f_local,
                                                         double *__restrict__ forces, ChunkSums cs) {
    constexpr int LPA = 8, NG = NT / LPA;
    const int c = blockIdx.x;
    const int s = cs.chunk[3 * c], a0 = cs.chunk[3 * c + 1], a1 = cs.chunk[3 * c + 2];
    const int sub = threadIdx.x & (LPA - 1), grp = threadIdx.x / LPA;
    double r0 = 0.0, r1 = 0.0;
    int nb = 0, ne = 0;
    if (a0 + grp < a1) {
        nb = row_off[a0 + grp];
        ne = row_off[a0 + grp + 1];
    }
    for (int base = a0; base < a1; base += NG) {  // uniform over the block
        const int a = base + grp, beg = nb, end = ne;
        if (a + NG < a1) {
            nb = row_off[a + NG];
            ne = row_off[a + NG + 1];
        }
        double fx = 0, fy = 0, fz = 0;
        if (a < a1) {
            // each slot force is read once: streaming (evict-first) loads
#pragma unroll 4
            for (int q = beg + sub; q < end; q += LPA) {
                fx += __ldcs(G + 3 * (size_t)q);
                fy += __ldcs(G + 3 * (size_t)q + 1);
                fz += __ldcs(G + 3 * (size_t)q + 2);
            }
            const double *pa = cs.per_atom + (size_t)a * ATOM_ACC;
            r0 += pa[sub];
            if (sub < ATOM_ACC - LPA) r1 += pa[LPA + sub];
        }
        fx = group_sum<LPA>(fx);
        fy = group_sum<LPA>(fy);
        fz = group_sum<LPA>(fz);
        if (sub == 0 && a < a1) {
            forces[3 * (size_t)a] = f_local[3 * (size_t)a] + fx;
            forces[3 * (size_t)a + 1] = f_local[3 * (size_t)a + 1] + fy;
            forces[3 * (size_t)a + 2] = f_local[3 * (size_t)a + 2] + fz;
        }
    }
    chunk_sums_finish<NT>(cs, c, s, r0, r1);
}

int gather_reduce(int n_struct, int n_atoms, const int *row_off, const double *G, const double *f_local,
                  double *forces, const double *per_atom, const mbf_reduce_plan *plan, double *partial,
                  double *energy, double *virial, unsigned *sdone, cudaStream_t st) {
    // the completion counters live in a region of n_chunks words; every
    // structure owns at least one chunk
    if (plan->n_chunks <= 0 || n_struct <= 0 || plan->n_chunks < n_struct || !sdone) return MBF_ERR_ARGUMENT;
    if (cudaMemsetAsync(sdone, 0, sizeof(unsigned) * (size_t)n_struct, st) != cudaSuccess) return MBF_ERR_CUDA;
    ChunkSums cs = {plan->chunk, plan->chunk_first, per_atom, partial, energy, virial, sdone};
    PROF_BEGIN("gather_reduce", st);
    int nt = chunk_block(n_atoms, plan->n_chunks);
    if (nt == 128)
        gather_reduce_rows<128><<<plan->n_chunks, 128, 0, st>>>(row_off, G, f_local, forces, cs);
    else if (nt == 256)
        gather_reduce_rows<256><<<plan->n_chunks, 256, 0, st>>>(row_off, G, f_local, forces, cs);
    else
        gather_reduce_rows<512><<<plan->n_chunks, 512, 0, st>>>(row_off, G, f_local, forces, cs);
    PROF_END("gather_reduce", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

}  // namespace mbf

extern "C" {

const char *mbf_error_string(int code) {
    switch (code) {
        case MBF_OK: return "ok";
        case MBF_ERR_ARGUMENT: return "invalid argument";
        case MBF_ERR_CUDA: return "CUDA runtime error";
        case MBF_ERR_CAPACITY: return "neighbour capacity too small";
        case MBF_ERR_ROW_TOO_LONG: return "neighbour row longer than the kernel's staging limit";
        case MBF_ERR_WORKSPACE: return "workspace too small";
        case MBF_ERR_SCRATCH_LIMIT: return "size beyond the no-allocation entry point's limit";
        default: return "unknown error";
    }
}

int mbf_version(void) { return 10000; }

size_t mbf_eval_workspace_bytes(int n_atoms, long long n_slots, int n_chunks) {
    return mbf::eval_layout(n_atoms, n_slots, n_chunks).total;
}

int mbf_eval_status(const void *workspace, int *host_words, void *stream) {
    if (!workspace || !host_words) return MBF_ERR_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(host_words, workspace, 4 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MBF_ERR_CUDA;
    return MBF_OK;
}

}  // extern "C"
