// Cell-list neighbour list: binning by integer counting sort, two-way CSR
// by count -> scan -> fill, rows sorted ascending, reverse-slot index.
//
// Replaces engine/neighborlist.py:935-1024 (_build_cell_linked), :312-373
// (_cell_linked_pairs_numpy), :1166-1181 (_canonical_pair_order) and the
// two-way CSR of engine/tersoff.py:1297-1307.  The pair test reproduces the
// reference's rounding exactly (mic_exact), so the pair set is bit-exact.
#include <type_traits>

#include "mbf_util.cuh"

namespace mbf {

constexpr int NL_WARPS = 4;        // warps per block in the search kernels
constexpr int NL_MAXROW = 1024;    // longest row the sort stages in shared memory

struct NlLayout {
    size_t err, atom_cell, cell_count, cell_start, cursor, cell_atoms, row_cnt, maxrow, scan, total;
};

static NlLayout nl_layout(int n_atoms, int n_cells) {
    NlLayout L;
    size_t o = 0;
    L.err = o;
    o = align256(o + 64);
    L.atom_cell = o;
    o = align256(o + sizeof(int) * (size_t)n_atoms);
    L.cell_count = o;
    o = align256(o + sizeof(int) * (size_t)n_cells);
    L.cell_start = o;
    o = align256(o + sizeof(int) * ((size_t)n_cells + 1));
    L.cursor = o;
    o = align256(o + sizeof(int) * (size_t)n_cells);
    L.cell_atoms = o;
    o = align256(o + sizeof(int) * (size_t)n_atoms);
    L.row_cnt = o;
    o = align256(o + sizeof(int) * (size_t)n_atoms);
    L.maxrow = o;
    o = align256(o + 64);
    L.scan = o;
    int nmax = n_atoms > n_cells ? n_atoms : n_cells;
    o = align256(o + sizeof(int) * scan_workspace_ints(nmax + 1));
    L.total = o;
    return L;
}

// The rebuild's staging rows (n_atoms x max_row_limit ints) after the layout.
static size_t nl_staged_bytes(const NlLayout &L, int n_atoms, int max_row_limit) {
    return L.total + align256(sizeof(int) * (size_t)n_atoms * (size_t)max_row_limit);
}

// Bin every atom: fractional coordinate wrapped to [0, 1), sub-cell index
// floor(frac * nc) clipped to [0, nc - 1] (engine/neighborlist.py:982-989).
__global__ void nl_assign(SysView S, const int *__restrict__ grids, int *__restrict__ atom_cell,
                          int *__restrict__ cell_count) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= S.n_atoms) return;
    int s = S.n_struct > 1 ? S.atom_struct[a] : 0;
    const int *g = grids + 8 * s;
    const double *inv = S.cells + 18 * (size_t)s + 9;
    double x = S.pos[3 * (size_t)a], y = S.pos[3 * (size_t)a + 1], z = S.pos[3 * (size_t)a + 2];
    int ci[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double f = x * inv[k] + y * inv[3 + k] + z * inv[6 + k];
        f = f - floor(f);
        int c = (int)floor(f * (double)g[k]);
        c = c < 0 ? 0 : (c > g[k] - 1 ? g[k] - 1 : c);
        ci[k] = c;
    }
    int cell = g[3] + (ci[0] * g[1] + ci[1]) * g[2] + ci[2];
    atom_cell[a] = cell;
    atomicAdd(cell_count + cell, 1);
}

__global__ void nl_fill_cells(int n_atoms, const int *__restrict__ atom_cell, int *__restrict__ cursor,
                              int *__restrict__ cell_atoms) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    int p = atomicAdd(cursor + atom_cell[a], 1);
    cell_atoms[p] = a;
}

// Stencil of atom a's cell: up to 27 neighbour cells (per-axis offsets
// {0} for nc = 1, {0, 1} for nc = 2, {-1, 0, 1} otherwise -- the reference's
// _axis_offsets, engine/neighborlist.py:270-299), visited in (da, db, dc)
// order.  Lane k < K describes cell k; returns the warp-wide candidate count.
struct Stencil {
    int start[32];
    int pre[33];
};

__device__ int build_stencil_of_cell(const int *__restrict__ grids, const int *__restrict__ cell_start,
                                     int s, int cell_id, Stencil &st) {
    int lane = threadIdx.x & 31;
    const int *g = grids + 8 * s;
    int nc0 = g[0], nc1 = g[1], nc2 = g[2], first = g[3];
    int w0 = g[4], w1 = g[5], w2 = g[6];
    int local = cell_id - first;
    int c2 = local % nc2, c1 = (local / nc2) % nc1, c0 = local / (nc1 * nc2);
    int K = w0 * w1 * w2;
    int len = 0, start = 0;
    if (lane < K) {
        int i0 = lane / (w1 * w2), i1 = (lane / w2) % w1, i2 = lane % w2;
        int o0 = w0 == 3 ? i0 - 1 : i0, o1 = w1 == 3 ? i1 - 1 : i1, o2 = w2 == 3 ? i2 - 1 : i2;
        int j0 = (c0 + o0 + nc0) % nc0, j1 = (c1 + o1 + nc1) % nc1, j2 = (c2 + o2 + nc2) % nc2;
        int cell = first + (j0 * nc1 + j1) * nc2 + j2;
        start = cell_start[cell];
        len = cell_start[cell + 1] - start;
    }
    int inc = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(MBF_FULL, inc, o);
        if (lane >= o) inc += t;
    }
    st.start[lane] = start;
    st.pre[lane] = inc - len;
    int total = __shfl_sync(MBF_FULL, inc, 31);
    if (lane == 0) st.pre[32] = total;
    __syncwarp();
    return total;
}

// Candidate t of the stencil -> atom index (binary search over the prefix).
__device__ __forceinline__ int stencil_atom(const Stencil &st, const int *__restrict__ cell_atoms, int t) {
    int lo = 0, hi = 31;
    while (lo < hi) {  // largest k with pre[k] <= t
        int mid = (lo + hi + 1) >> 1;
        if (st.pre[mid] <= t) lo = mid; else hi = mid - 1;
    }
    // skip empty cells that share the same prefix value
    return cell_atoms[st.start[lo] + (t - st.pre[lo])];
}

// ---- warp per cell -----------------------------------------------------------
// The atoms of one cell share their stencil: a warp builds it once, each lane
// loads one candidate's position per round, and the cell's atoms (32 at a
// time, one per lane) are broadcast by shuffles and tested against every
// lane's candidate.  A pair (a, b != a) is listed iff r2 < r_list^2 and
// r2 > 1e-20, r2 from mic_exact of r_b - r_a: the reference's test in its
// own operation order (engine/neighborlist.py:350-363).
__device__ __forceinline__ bool pair_hit(const double *__restrict__ cell, double xa, double ya, double za,
                                         double xb, double yb, double zb, double rl2) {
    double dx, dy, dz;
    mic_exact(cell, xb - xa, yb - ya, zb - za, dx, dy, dz);
    double r2 = r2_exact(dx, dy, dz);
    return r2 < rl2 && r2 > 1e-20;
}

// A cell whose lattice and inverse have exact zeros off the diagonal.
__device__ __forceinline__ bool cell_is_diagonal(const double *__restrict__ c) {
    bool z = true;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const double *q = c + 9 * m;
        z = z && q[1] == 0.0 && q[2] == 0.0 && q[3] == 0.0 && q[5] == 0.0 && q[6] == 0.0 && q[7] == 0.0;
    }
    return z;
}

// pair_hit for a diagonal cell (d = inverse diagonal, l = lattice
// diagonal).  Each dropped term of mic_exact's dot products is a product
// with an exact zero, i.e. +-0, and x + (+-0) == x for every x != 0, so
// every component equals mic_exact's up to the sign of a zero, and r2 --
// a sum of squares -- is the same double bit for bit.
__device__ __forceinline__ bool pair_hit_diag(double d0, double d1, double d2, double l0, double l1, double l2,
                                              double xa, double ya, double za, double xb, double yb, double zb,
                                              double rl2) {
    double sx = __dmul_rn(__dsub_rn(xb, xa), d0);
    double sy = __dmul_rn(__dsub_rn(yb, ya), d1);
    double sz = __dmul_rn(__dsub_rn(zb, za), d2);
    sx = __dsub_rn(sx, rint_shift(sx));
    sy = __dsub_rn(sy, rint_shift(sy));
    sz = __dsub_rn(sz, rint_shift(sz));
    double r2 = r2_exact(__dmul_rn(sx, l0), __dmul_rn(sy, l1), __dmul_rn(sz, l2));
    return r2 < rl2 && r2 > 1e-20;
}

// MODE 0 counts each atom's neighbours (row_cnt, max_row); MODE 1 writes
// them into the CSR rows (row_off, nbr); MODE 2 counts and writes them at a
// fixed stride into a staging array (`nbr` = stage, row a at a * stride,
// at most stride entries kept), so one pass serves a list of known row
// bound.
template <int MODE>
__global__ void nl_cells(SysView S, const int *__restrict__ grids, const int *__restrict__ cell_start,
                         const int *__restrict__ cell_atoms, int n_cells, double rl2, int *__restrict__ row_cnt,
                         int *__restrict__ max_row, const int *__restrict__ row_off, int *__restrict__ nbr,
                         int stride) {
    constexpr bool FILL = MODE != 0, COUNT = MODE != 1;
    __shared__ Stencil sst[NL_WARPS];
    int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Stencil &st = sst[wid];
    for (int c = blockIdx.x * NL_WARPS + wid; c < n_cells; c += gridDim.x * NL_WARPS) {
        int cs = cell_start[c], na = cell_start[c + 1] - cs;
        if (na == 0) continue;  // uniform over the warp
        int a0 = cell_atoms[cs];
        int sidx = S.n_struct > 1 ? S.atom_struct[a0] : 0;
        int total = build_stencil_of_cell(grids, cell_start, sidx, c, st);
        const double *cell = S.cells + 18 * (size_t)sidx;
        const bool diag = cell_is_diagonal(cell);
        const double d0 = cell[9], d1 = cell[13], d2 = cell[17], l0 = cell[0], l1 = cell[4], l2 = cell[8];
        for (int q0 = 0; q0 < na; q0 += 32) {
            int nq = min(32, na - q0);
            int a_l = lane < nq ? cell_atoms[cs + q0 + lane] : 0;
            double xa_l = S.pos[3 * (size_t)a_l], ya_l = S.pos[3 * (size_t)a_l + 1], za_l = S.pos[3 * (size_t)a_l + 2];
            int cnt = 0;       // lane q: neighbours of atom q found so far
            int beg_l = 0, len_l = 0;
            if (FILL && lane < nq) {
                beg_l = MODE == 1 ? row_off[a_l] : a_l * stride;
                len_l = MODE == 1 ? row_off[a_l + 1] - beg_l : stride;
            }
            for (int t0 = 0; t0 < total; t0 += 32) {
                int t = t0 + lane;
                int b = -1;
                double xb = 0, yb = 0, zb = 0;
                if (t < total) {
                    b = stencil_atom(st, cell_atoms, t);
                    xb = S.pos[3 * (size_t)b];
                    yb = S.pos[3 * (size_t)b + 1];
                    zb = S.pos[3 * (size_t)b + 2];
                }
                // the cell's atoms against this round's candidates, with
                // the test specialised once per cell (warp-uniform)
                auto rounds = [&](auto diag_tag) {
                    constexpr bool DIAG = decltype(diag_tag)::value;
                    for (int q = 0; q < nq; ++q) {
                        int a = __shfl_sync(MBF_FULL, a_l, q);
                        double xa = __shfl_sync(MBF_FULL, xa_l, q), ya = __shfl_sync(MBF_FULL, ya_l, q),
                               za = __shfl_sync(MBF_FULL, za_l, q);
                        bool hit = b >= 0 && b != a &&
                                   (DIAG ? pair_hit_diag(d0, d1, d2, l0, l1, l2, xa, ya, za, xb, yb, zb, rl2)
                                         : pair_hit(cell, xa, ya, za, xb, yb, zb, rl2));
                        unsigned m = __ballot_sync(MBF_FULL, hit);
                        if (FILL) {
                            int w = __shfl_sync(MBF_FULL, cnt, q);
                            int beg = __shfl_sync(MBF_FULL, beg_l, q), len = __shfl_sync(MBF_FULL, len_l, q);
                            if (hit) {
                                int pos = w + __popc(m & ((1u << lane) - 1u));
                                if (pos < len) nbr[beg + pos] = b;
                            }
                        }
                        if (lane == q) cnt += __popc(m);
                    }
                };
                if (diag)
                    rounds(std::true_type{});
                else
                    rounds(std::false_type{});
            }
            if (COUNT && lane < nq) {
                row_cnt[a_l] = cnt;
                atomicMax(max_row, cnt);
            }
        }
    }
}

// ---- row sorts -----------------------------------------------------------------
// Rows come out of the search in traversal order; the CSR keeps them
// ascending.  By length n: up to 32 entries one per lane, ranked by
// shuffles; up to 64 or 128 a bitonic network in registers over J = 2 or 4
// entries a lane (entry e = J lane + j, padded with INT_MAX, which sorts
// last since atom indices are smaller); longer rows by rank in shared
// memory.  Entries of a row are distinct.
constexpr int NL_PAD = 0x7fffffff;

__device__ __forceinline__ void cmp_swap(int &lo, int &hi, bool asc) {
    int mn = min(lo, hi), mx = max(lo, hi);
    lo = asc ? mn : mx;
    hi = asc ? mx : mn;
}

template <int J>
__device__ __forceinline__ void bitonic_sort(int (&v)[J]) {
    int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32 * J; k <<= 1) {
#pragma unroll
        for (int d = k >> 1; d > 0; d >>= 1) {
            if (d >= J) {  // partner in lane ^ (d / J), same register
                bool low = (lane & (d / J)) == 0;
#pragma unroll
                for (int j = 0; j < J; ++j) {
                    int o = __shfl_xor_sync(MBF_FULL, v[j], d / J);
                    bool asc = ((J * lane + j) & k) == 0;
                    v[j] = (low == asc) ? min(v[j], o) : max(v[j], o);
                }
            } else {  // partner in register j ^ d of this lane
#pragma unroll
                for (int j = 0; j < J; ++j)
                    if ((j & d) == 0) cmp_swap(v[j], v[j ^ d], ((J * lane + j) & k) == 0);
            }
        }
    }
}

// Sorts n <= 32 J entries src[0..n) into out[0..n); returns this lane's
// count of entries below `a`.
template <int J>
__device__ __forceinline__ int sort_row_bitonic(const int *src, int n, int *out, int a) {
    int lane = threadIdx.x & 31;
    int v[J];
#pragma unroll
    for (int j = 0; j < J; ++j) v[j] = J * lane + j < n ? src[J * lane + j] : NL_PAD;
    __syncwarp();
    bitonic_sort<J>(v);
    int lower = 0;
#pragma unroll
    for (int j = 0; j < J; ++j)
        if (J * lane + j < n) {
            out[J * lane + j] = v[j];
            lower += v[j] < a ? 1 : 0;
        }
    return lower;
}

// Sorts the n entries src[0..n) (n <= NL_MAXROW) ascending into out[0..n)
// (src and out may be the same row: every entry is read before any is
// written) and returns how many are below `a` (warp-uniform).  `row` is
// the warp's shared scratch of NL_MAXROW ints.
__device__ __forceinline__ int sort_row(const int *src, int n, int *out, int a, int *row) {
    int lane = threadIdx.x & 31;
    int lower = 0;
    if (n <= 32) {
        int v = lane < n ? src[lane] : NL_PAD, rank = 0;
        for (int q = 0; q < n; ++q) rank += __shfl_sync(MBF_FULL, v, q) < v ? 1 : 0;
        if (lane < n) {
            out[rank] = v;
            lower = v < a ? 1 : 0;
        }
    } else if (n <= 64) {
        lower = sort_row_bitonic<2>(src, n, out, a);
    } else if (n <= 128) {
        lower = sort_row_bitonic<4>(src, n, out, a);
    } else {
        for (int k = lane; k < n; k += 32) row[k] = src[k];
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
            int v = row[k], rank = 0;
            for (int q = 0; q < n; ++q) rank += row[q] < v ? 1 : 0;
            out[rank] = v;
            lower += v < a ? 1 : 0;
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lower += __shfl_xor_sync(MBF_FULL, lower, o);
    return lower;
}

// Each cell's atoms in ascending index order, so the traversal (and the
// rows it produces) do not depend on the order of nl_fill_cells's atomics:
// a warp per cell, the row sort above (a cell beyond NL_MAXROW atoms, which
// no physical density reaches, by insertion on one lane).
__global__ void nl_sort_cells(int n_cells, const int *__restrict__ cell_start, int *__restrict__ cell_atoms) {
    __shared__ int srow[NL_WARPS][NL_MAXROW];
    int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x * NL_WARPS + wid; c < n_cells; c += gridDim.x * NL_WARPS) {
        int b = cell_start[c], n = cell_start[c + 1] - b;
        if (n <= NL_MAXROW) {
            sort_row(cell_atoms + b, n, cell_atoms + b, NL_PAD, srow[wid]);
        } else if (lane == 0) {
            for (int i = b + 1; i < b + n; ++i) {
                int v = cell_atoms[i];
                int j = i - 1;
                while (j >= b && cell_atoms[j] > v) {
                    cell_atoms[j + 1] = cell_atoms[j];
                    --j;
                }
                cell_atoms[j + 1] = v;
            }
        }
        __syncwarp();
    }
}

// Rows written in traversal order by nl_cells<1>: sorted in place, and
// each row's first upper slot recorded.
__global__ void nl_sort_rows(int n_atoms, const int *__restrict__ row_off, int *__restrict__ nbr,
                             int *__restrict__ upper, int *__restrict__ err) {
    __shared__ int srow[NL_WARPS][NL_MAXROW];
    int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int a = blockIdx.x * NL_WARPS + wid; a < n_atoms; a += gridDim.x * NL_WARPS) {
        int beg = row_off[a], n = row_off[a + 1] - beg;
        if (n > NL_MAXROW) {
            if (lane == 0) {
                atomicOr(err, MBF_DEV_ROW_TOO_LONG);
                upper[a] = beg;
            }
            continue;
        }
        int lower = sort_row(nbr + beg, n, nbr + beg, a, srow[wid]);
        if (lane == 0) upper[a] = beg + lower;
    }
}

// The staged rows (nl_cells<2>) into the CSR: each row read from its
// stride-spaced staging slot, sorted and written at its scanned offset;
// its first upper slot recorded.  Rows longer than the stride were refused
// by the guard (their rows are empty by then).
__global__ void nl_unstage_rows(int n_atoms, const int *__restrict__ row_off, const int *__restrict__ stage,
                                int stride, int *__restrict__ nbr, int *__restrict__ upper, int *__restrict__ err) {
    __shared__ int srow[NL_WARPS][NL_MAXROW];
    int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int a = blockIdx.x * NL_WARPS + wid; a < n_atoms; a += gridDim.x * NL_WARPS) {
        int beg = row_off[a], n = row_off[a + 1] - beg;
        if (n > stride || n > NL_MAXROW) {
            if (lane == 0) {
                atomicOr(err, MBF_DEV_ROW_TOO_LONG);
                upper[a] = beg;
            }
            continue;
        }
        int lower = sort_row(stage + (size_t)a * stride, n, nbr + beg, a, srow[wid]);
        if (lane == 0) upper[a] = beg + lower;
    }
}

// Reverse slot of every slot.  rev is an involution, so only the upper
// slots (a -> b, b > a) search: a lies in the lower part of b's sorted row,
// [row_off[b], upper[b]); the slot t found there gets rev[t] = s, so every
// slot is written once.  Eight lanes per row: an upper part holds about
// half a row, so short rows keep the lanes busy.
constexpr int NL_REV_LANES = 8;

__global__ void nl_reverse(int n_atoms, const int *__restrict__ row_off, const int *__restrict__ upper,
                           const int *__restrict__ nbr, int *__restrict__ rev, int *__restrict__ err) {
    const int grp = threadIdx.x / NL_REV_LANES, sub = threadIdx.x % NL_REV_LANES;
    const int per_block = 32 * NL_WARPS / NL_REV_LANES;
    for (int a = blockIdx.x * per_block + grp; a < n_atoms; a += gridDim.x * per_block) {
        for (int s = upper[a] + sub; s < row_off[a + 1]; s += NL_REV_LANES) {
            int b = nbr[s];
            int lo = row_off[b], hi = upper[b] - 1, found = -1;
            while (lo <= hi) {
                int mid = (lo + hi) >> 1;
                int v = nbr[mid];
                if (v == a) { found = mid; break; }
                if (v < a) lo = mid + 1; else hi = mid - 1;
            }
            if (found < 0) {
                atomicOr(err, MBF_DEV_BAD_INDEX);
                rev[s] = s;
                continue;
            }
            rev[s] = found;
            rev[found] = s;
        }
    }
}

// Per-structure largest minimum-image displacement from the reference
// positions mapped by the lattice change (engine/neighborlist.py:661-668).
__global__ void nl_max_disp(SysView S, const double *__restrict__ ref, const double *__restrict__ maps,
                            unsigned long long *__restrict__ dmax_bits) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= S.n_atoms) return;
    int s = S.n_struct > 1 ? S.atom_struct[a] : 0;
    const double *r0 = ref + 3 * (size_t)a;
    double ax = r0[0], ay = r0[1], az = r0[2];
    if (maps) {  // null: lattice unchanged, M = I
        const double *M = maps + 9 * (size_t)s;
        ax = r0[0] * M[0] + r0[1] * M[3] + r0[2] * M[6];
        ay = r0[0] * M[1] + r0[1] * M[4] + r0[2] * M[7];
        az = r0[0] * M[2] + r0[1] * M[5] + r0[2] * M[8];
    }
    double dx, dy, dz;
    mic_exact(S.cells + 18 * (size_t)s, S.pos[3 * (size_t)a] - ax, S.pos[3 * (size_t)a + 1] - ay,
              S.pos[3 * (size_t)a + 2] - az, dx, dy, dz);
    double d = sqrt(dx * dx + dy * dy + dz * dz);
    atomicMax(dmax_bits + s, (unsigned long long)__double_as_longlong(d));
}

__global__ void nl_upper_count(int n_atoms, const int *__restrict__ row_off, const int *__restrict__ nbr,
                               int *__restrict__ up) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    int c = 0;
    for (int s = row_off[a]; s < row_off[a + 1]; ++s) c += nbr[s] > a ? 1 : 0;
    up[a] = c;
}

__global__ void nl_upper_write(int n_atoms, const int *__restrict__ row_off, const int *__restrict__ nbr,
                               const int *__restrict__ up_off, int *__restrict__ pi, int *__restrict__ pj) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    int o = up_off[a];
    for (int s = row_off[a]; s < row_off[a + 1]; ++s) {
        int b = nbr[s];
        if (b > a) {
            pi[o] = a;
            pj[o] = b;
            ++o;
        }
    }
}

// Device-side checks of the graph-capturable rebuild: a list that would not
// fit its buffers or a row beyond the caller's staging limit sets a status
// bit and leaves every row empty (no slot is written), so later kernels of a
// captured sequence read nothing out of bounds.
__global__ void nl_guard(int n_atoms, const int *__restrict__ row_off, const int *__restrict__ mrow,
                         long long cap, int limit, int *__restrict__ status, int *__restrict__ skip) {
    if (threadIdx.x != 0) return;
    int bad = 0;
    if ((long long)row_off[n_atoms] > cap) bad |= MBF_STATUS_CAPACITY;
    if (*mrow > limit) bad |= MBF_STATUS_ROW_TOO_LONG;
    *skip = bad;
    if (bad) atomicOr(status, bad);
}

__global__ void nl_clear_if(int n_atoms, const int *__restrict__ skip, int *__restrict__ row_off,
                            int *__restrict__ upper) {
    if (*skip == 0) return;
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a <= n_atoms) row_off[a] = 0;
    if (a < n_atoms) upper[a] = 0;
}

// Records d (this step's largest displacement since the last rebuild) and
// the reference's rebuild decision r_list - 2 d <= r_cut (any structure,
// engine/neighborlist.py:653-673 with the lattice unchanged); sets the
// graph conditional that gates the rebuild branch when one is given, and
// flags MBF_STATUS_SKIN when a status word is given (fixed-interval runs,
// where the decision is an assertion).
__global__ void nl_skin_record(int n_struct, const double *__restrict__ d, double r_list, double r_cut,
                               double *__restrict__ d_log,
                               int rows, int *__restrict__ counter, int *__restrict__ gate, int *__restrict__ status,
                               unsigned long long cond) {
    if (threadIdx.x != 0) return;
    int row = *counter % rows;
    int need = 0;
    for (int s = 0; s < n_struct; ++s) {
        d_log[(size_t)row * n_struct + s] = d[s];
        if (r_list - 2.0 * d[s] <= r_cut) need = 1;
    }
    *gate = need;
    if (need && status) atomicOr(status, MBF_STATUS_SKIN);
    if (cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, need ? 1u : 0u);
    *counter += 1;
}

__global__ void nl_count_rebuild(int *__restrict__ n) {
    if (threadIdx.x == 0) *n += 1;
}

__global__ void nl_status_merge(const int *__restrict__ err, int *__restrict__ status) {
    if (threadIdx.x != 0) return;
    int e = err[0];
    if (e & MBF_DEV_ROW_TOO_LONG) atomicOr(status, MBF_STATUS_ROW_TOO_LONG);
    if (e & ~MBF_DEV_ROW_TOO_LONG) atomicOr(status, MBF_STATUS_BAD_INDEX);
}

}  // namespace mbf

using namespace mbf;

extern "C" {

size_t mbf_nl_workspace_bytes(int n_atoms, int n_cells_total) {
    return nl_layout(n_atoms, n_cells_total).total;
}

size_t mbf_nl_rebuild_workspace_bytes(int n_atoms, int n_cells_total, int max_row_limit) {
    if (n_atoms < 0 || n_cells_total <= 0 || max_row_limit <= 0) return 0;
    return nl_staged_bytes(nl_layout(n_atoms, n_cells_total), n_atoms, max_row_limit);
}

static int nl_prepare(const SysView &S, const int *grids, int n_cells_total, double rl2, void *workspace,
                      const NlLayout &L, int *row_off, cudaStream_t st, int *stage = nullptr, int stride = 0) {
    int N = S.n_atoms;
    int *err = ws_at<int>(workspace, L.err);
    int *atom_cell = ws_at<int>(workspace, L.atom_cell);
    int *cell_count = ws_at<int>(workspace, L.cell_count);
    int *cell_start = ws_at<int>(workspace, L.cell_start);
    int *cursor = ws_at<int>(workspace, L.cursor);
    int *cell_atoms = ws_at<int>(workspace, L.cell_atoms);
    int *row_cnt = ws_at<int>(workspace, L.row_cnt);
    int *mrow = ws_at<int>(workspace, L.maxrow);
    int *scan_ws = ws_at<int>(workspace, L.scan);
    if (cudaMemsetAsync(err, 0, 64, st) != cudaSuccess) return MBF_ERR_CUDA;
    if (cudaMemsetAsync(mrow, 0, sizeof(int), st) != cudaSuccess) return MBF_ERR_CUDA;
    if (cudaMemsetAsync(cell_count, 0, sizeof(int) * (size_t)n_cells_total, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    PROF_BEGIN("nl_assign", st);
    nl_assign<<<(N + 255) / 256, 256, 0, st>>>(S, grids, atom_cell, cell_count);
    PROF_END("nl_assign", st);
    MBF_CHECK_LAUNCH();
    int rc = exclusive_scan(cell_count, cell_start, n_cells_total, scan_ws, st);
    if (rc != MBF_OK) return rc;
    if (cudaMemcpyAsync(cursor, cell_start, sizeof(int) * (size_t)n_cells_total,
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    nl_fill_cells<<<(N + 255) / 256, 256, 0, st>>>(N, atom_cell, cursor, cell_atoms);
    nl_sort_cells<<<persistent_grid((n_cells_total + NL_WARPS - 1) / NL_WARPS, 32 * NL_WARPS,
                                    (const void *)nl_sort_cells),
                    32 * NL_WARPS, 0, st>>>(n_cells_total, cell_start, cell_atoms);
    MBF_CHECK_LAUNCH();
    int cblocks = (n_cells_total + NL_WARPS - 1) / NL_WARPS;
    int g = persistent_grid(cblocks, 32 * NL_WARPS, (const void *)nl_cells<0>);
    PROF_BEGIN("nl_count", st);
    if (stage) {
        g = persistent_grid(cblocks, 32 * NL_WARPS, (const void *)nl_cells<2>);
        nl_cells<2><<<g, 32 * NL_WARPS, 0, st>>>(S, grids, cell_start, cell_atoms, n_cells_total, rl2, row_cnt, mrow,
                                                 nullptr, stage, stride);
    } else {
        nl_cells<0><<<g, 32 * NL_WARPS, 0, st>>>(S, grids, cell_start, cell_atoms, n_cells_total, rl2, row_cnt, mrow,
                                                 nullptr, nullptr, 0);
    }
    PROF_END("nl_count", st);
    MBF_CHECK_LAUNCH();
    return exclusive_scan(row_cnt, row_off, N, scan_ws, st);
}

static int nl_finish(const SysView &S, const int *grids, int n_cells_total, double rl2, void *workspace,
                     const NlLayout &L, const int *row_off, int *nbr, int *rev, int *upper, cudaStream_t st,
                     const int *stage = nullptr, int stride = 0) {
    int N = S.n_atoms;
    int *err = ws_at<int>(workspace, L.err);
    int blocks = (N + NL_WARPS - 1) / NL_WARPS;
    int cblocks = (n_cells_total + NL_WARPS - 1) / NL_WARPS;
    int g = persistent_grid(cblocks, 32 * NL_WARPS, (const void *)nl_cells<1>);
    PROF_BEGIN("nl_fill", st);
    if (stage) {
        g = persistent_grid(blocks, 32 * NL_WARPS, (const void *)nl_unstage_rows);
        nl_unstage_rows<<<g, 32 * NL_WARPS, 0, st>>>(N, row_off, stage, stride, nbr, upper, err);
    } else {
        nl_cells<1><<<g, 32 * NL_WARPS, 0, st>>>(S, grids, ws_at<int>(workspace, L.cell_start),
                                                 ws_at<int>(workspace, L.cell_atoms), n_cells_total, rl2, nullptr,
                                                 nullptr, row_off, nbr, 0);
        g = persistent_grid(blocks, 32 * NL_WARPS, (const void *)nl_sort_rows);
        nl_sort_rows<<<g, 32 * NL_WARPS, 0, st>>>(N, row_off, nbr, upper, err);
    }
    PROF_END("nl_fill", st);
    MBF_CHECK_LAUNCH();
    g = persistent_grid((N + 32 * NL_WARPS / NL_REV_LANES - 1) / (32 * NL_WARPS / NL_REV_LANES), 32 * NL_WARPS,
                        (const void *)nl_reverse);
    PROF_BEGIN("nl_reverse", st);
    nl_reverse<<<g, 32 * NL_WARPS, 0, st>>>(N, row_off, upper, nbr, rev, err);
    PROF_END("nl_reverse", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_nl_build(const mbf_system *sys, const int *grids, int n_cells_total, double r_list,
                 void *workspace, size_t workspace_bytes, int *row_off, int *nbr, int *rev, int *upper,
                 long long nbr_capacity, long long *n_slots, int *max_row, void *stream) {
    if (!sys || !grids || !workspace || !row_off || !n_slots || !max_row || sys->n_atoms < 0 ||
        n_cells_total <= 0 || !(r_list > 0.0))
        return MBF_ERR_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    int N = sys->n_atoms;
    NlLayout L = nl_layout(N, n_cells_total);
    if (workspace_bytes < L.total) return MBF_ERR_WORKSPACE;
    SysView S = make_view(sys);
    if (N == 0) {
        if (cudaMemsetAsync(row_off, 0, sizeof(int), st) != cudaSuccess) return MBF_ERR_CUDA;
        *n_slots = 0;
        *max_row = 0;
        return MBF_OK;
    }
    double rl2 = r_list * r_list;
    // workspace beyond the layout holds staging rows at the stride it allows:
    // if no row is longer, the search runs once (count and stage, then sort
    // into the CSR), else the rows are searched again (fill)
    int stride = 0;
    if (workspace_bytes >= L.total + 256) {
        size_t per = (workspace_bytes - L.total) / (sizeof(int) * (size_t)N);
        stride = (int)(per < (size_t)NL_MAXROW ? per : (size_t)NL_MAXROW);
        if ((long long)N * stride >= 0x7fffffffLL) stride = (int)(0x7ffffffeLL / N);
    }
    int *stage = stride > 0 ? ws_at<int>(workspace, L.total) : nullptr;
    int rc = nl_prepare(S, grids, n_cells_total, rl2, workspace, L, row_off, st, stage, stride);
    if (rc != MBF_OK) return rc;
    int host[2];
    if (cudaMemcpyAsync(&host[0], row_off + N, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&host[1], ws_at<int>(workspace, L.maxrow), sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MBF_ERR_CUDA;
    *n_slots = host[0];
    *max_row = host[1];
    if ((long long)host[0] > nbr_capacity || !nbr || !rev) return MBF_ERR_CAPACITY;
    if (!upper) return MBF_ERR_ARGUMENT;
    if (host[1] > NL_MAXROW) return MBF_ERR_ROW_TOO_LONG;
    if (host[1] > stride) stage = nullptr;
    rc = nl_finish(S, grids, n_cells_total, rl2, workspace, L, row_off, nbr, rev, upper, st, stage,
                   stage ? stride : 0);
    if (rc != MBF_OK) return rc;
    int herr = 0;
    if (cudaMemcpyAsync(&herr, ws_at<int>(workspace, L.err), sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MBF_ERR_CUDA;
    if (herr & MBF_DEV_ROW_TOO_LONG) return MBF_ERR_ROW_TOO_LONG;
    if (herr) return MBF_ERR_ARGUMENT;
    return MBF_OK;
}

int mbf_nl_rebuild_async(const mbf_system *sys, const int *grids, int n_cells_total, double r_list,
                         void *workspace, size_t workspace_bytes, int *row_off, int *nbr, int *rev, int *upper,
                         long long nbr_capacity, int max_row_limit, int *status, void *stream) {
    if (!sys || !grids || !workspace || !row_off || !nbr || !rev || !upper || !status || sys->n_atoms <= 0 ||
        n_cells_total <= 0 || !(r_list > 0.0) || nbr_capacity < 0 || max_row_limit <= 0 ||
        max_row_limit > NL_MAXROW)
        return MBF_ERR_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    int N = sys->n_atoms;
    NlLayout L = nl_layout(N, n_cells_total);
    if (workspace_bytes < L.total) return MBF_ERR_WORKSPACE;
    SysView S = make_view(sys);
    double rl2 = r_list * r_list;
    // with room for the staging rows the search runs once (count and stage),
    // else it counts, then fills
    int *stage = nullptr;
    if (workspace_bytes >= nl_staged_bytes(L, N, max_row_limit) && (long long)N * max_row_limit < 0x7fffffffLL)
        stage = ws_at<int>(workspace, L.total);
    int rc = nl_prepare(S, grids, n_cells_total, rl2, workspace, L, row_off, st, stage, max_row_limit);
    if (rc != MBF_OK) return rc;
    int *err = ws_at<int>(workspace, L.err);
    nl_guard<<<1, 32, 0, st>>>(N, row_off, ws_at<int>(workspace, L.maxrow), nbr_capacity, max_row_limit, status,
                               err + 4);
    nl_clear_if<<<(N + 256) / 256, 256, 0, st>>>(N, err + 4, row_off, upper);
    MBF_CHECK_LAUNCH();
    rc = nl_finish(S, grids, n_cells_total, rl2, workspace, L, row_off, nbr, rev, upper, st, stage, max_row_limit);
    if (rc != MBF_OK) return rc;
    nl_status_merge<<<1, 32, 0, st>>>(err, status);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_nl_max_displacement(const mbf_system *sys, const double *ref_positions, const double *maps,
                            double *d_max, void *stream) {
    if (!sys || !ref_positions || !maps || !d_max) return MBF_ERR_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    SysView S = make_view(sys);
    if (cudaMemsetAsync(d_max, 0, sizeof(double) * (size_t)sys->n_struct, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    if (sys->n_atoms == 0) return MBF_OK;
    nl_max_disp<<<(sys->n_atoms + 255) / 256, 256, 0, st>>>(S, ref_positions, maps,
                                                            (unsigned long long *)d_max);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_md_skin_check(const mbf_system *sys, const double *ref_positions, double r_list, double r_cut,
                      double *d_scratch, double *d_log, int rows, int *counter, int *gate, int *status,
                      unsigned long long cond_handle, void *stream) {
    if (!sys || !ref_positions || !d_scratch || !d_log || !counter || !gate || rows <= 0 || !(r_list > r_cut) ||
        !(r_cut > 0.0) || sys->n_struct <= 0)
        return MBF_ERR_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    SysView S = make_view(sys);
    if (cudaMemsetAsync(d_scratch, 0, sizeof(double) * (size_t)sys->n_struct, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    if (sys->n_atoms > 0) {
        nl_max_disp<<<(sys->n_atoms + 255) / 256, 256, 0, st>>>(S, ref_positions, nullptr,
                                                                (unsigned long long *)d_scratch);
        MBF_CHECK_LAUNCH();
    }
    nl_skin_record<<<1, 32, 0, st>>>(sys->n_struct, d_scratch, r_list, r_cut, d_log, rows, counter, gate,
                                     status, cond_handle);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

int mbf_md_rebuild_done(const mbf_system *sys, double *ref_positions, int *rebuild_count, void *stream) {
    if (!sys || !ref_positions || !rebuild_count) return MBF_ERR_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    if (sys->n_atoms > 0 &&
        cudaMemcpyAsync(ref_positions, sys->positions, sizeof(double) * 3 * (size_t)sys->n_atoms,
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    nl_count_rebuild<<<1, 32, 0, st>>>(rebuild_count);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

size_t mbf_nl_half_workspace_bytes(int n_atoms) {
    return sizeof(int) * ((size_t)2 * n_atoms + 2 + scan_workspace_ints(n_atoms + 1)) + 256;
}

int mbf_nl_half_pairs(const mbf_nlist *nl, int *pair_i, int *pair_j, void *workspace,
                      size_t workspace_bytes, void *stream) {
    if (!nl || !pair_i || !pair_j || !workspace) return MBF_ERR_ARGUMENT;
    int N = nl->n_atoms;
    if (workspace_bytes < mbf_nl_half_workspace_bytes(N)) return MBF_ERR_WORKSPACE;
    if (N == 0) return MBF_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int *up = (int *)workspace;
    int *up_off = up + N;
    int *scan_ws = up_off + N + 2;
    nl_upper_count<<<(N + 255) / 256, 256, 0, st>>>(N, nl->row_off, nl->nbr, up);
    MBF_CHECK_LAUNCH();
    int rc = exclusive_scan(up, up_off, N, scan_ws, st);
    if (rc != MBF_OK) return rc;
    nl_upper_write<<<(N + 255) / 256, 256, 0, st>>>(N, nl->row_off, nl->nbr, up_off, pair_i, pair_j);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

}  // extern "C"
