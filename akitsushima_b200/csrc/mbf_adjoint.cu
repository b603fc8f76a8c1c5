// Tersoff adjoint: the vector-Jacobian product of (E, F, virial) with
// respect to the dense parameter tables, for fitting.
//
// With upstream gradients gE (per structure), gF (per atom) and gW (per
// structure, 3x3), the pull-back onto a parameter theta is
//
//   sum_s gE_s dE_s/dtheta + sum_a gF_a . dF_a/dtheta + sum_s gW_s : dW_s/dtheta
//     = d/dtheta [ sum_s gE_s E_s + D_t E ],
//
// because F_a = -dE/dr_a and W_ab = -dE/deps_ab (the virial of a homogeneous
// strain r -> (I + eps) r, compressive-positive stress times volume).  D_t E
// is the derivative of the energy along the tangent field that moves every
// pair vector d_ij (minimum image, j - i) by t_ij = gF_i - gF_j - gW d_ij.
//
// The energy is a sum of directed bond terms, each evaluated from centre i:
//   V_ij = 1/2 fc(r_ij) [fR(r_ij) + b_ij(zeta_ij) fA(r_ij)],
// summing to sum_{i<j} fc (fR + (b_ij + b_ji)/2 fA) (engine/tersoff.py:6-19,
// :1399-1414, with the multi-species gating and table reads of
// :1518-1711).  Every directed bond is re-evaluated here -- zeta included,
// no per-triplet intermediate is stored -- in hyper-dual arithmetic: one
// infinitesimal along the tangent t and K along parameter "sites" (the
// places a bond reads a table entry).  The cross term of (tangent, site p)
// is d(D_t V)/dtheta_p, the site part dV/dtheta_p.  Sites are reduced onto
// the table entries they read in a fixed order (deterministic).
//
// Sites of a bond (i, j) (W = 8 + 7 ns of them):
//   0..5   A, B, lambda1, lambda2, R, D of the pair record tb[lo, hi]
//   6, 7   beta, n of the centre's record tb[s_i, s_j]
//   8 + 7 s_k + 0..4  c, d, h, lambda3, gamma of tri[s_i, s_j, s_k]
//   8 + 7 s_k + 5, 6  R, D of tb[s_i, s_k] (the cutoff of leg i-k)
#include "mbf_hd.cuh"

namespace mbf {

constexpr int ADJ_K = 8;        // parameter directions per pass
constexpr int ADJ_BLOCK = 64;

// fc(r) = 1/2 - 1/2 sin(pi/2 (r - R)/D) on [R - D, R + D] (engine/tersoff.py:48-54).
template <int K>
__device__ __forceinline__ HD<K> hd_fc(const HD<K> &r, const HD<K> &R, const HD<K> &D) {
    if (r.v < R.v - D.v) return hd_const<K>(1.0);
    if (r.v > R.v + D.v) return hd_const<K>(0.0);
    HD<K> a = (0.5 * 3.14159265358979323846) * ((r - R) / D);
    return 0.5 + (-0.5) * hd_sin<K>(a);
}

// (lambda3 u)^m for m = 1 or 3; pow otherwise (m is not a fitted value).
template <int K>
__device__ __forceinline__ HD<K> hd_arg(const HD<K> &l3, const HD<K> &u, double m) {
    if (m == 3.0) return (l3 * l3 * l3) * (u * u * u);
    if (m == 1.0) return l3 * u;
    HD<K> mm = hd_const<K>(m);
    return hd_pow<K>(l3, mm) * hd_pow<K>(u, mm);
}

// The slot's owning atom: rows are sorted, so a binary search in row_off.
__device__ __forceinline__ int slot_owner(const int *__restrict__ row_off, int n_atoms, int s) {
    int lo = 0, hi = n_atoms - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (row_off[mid] <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}

struct AdjTab {
    int ns;
    const double *tb;   // (ns*ns, 10): valid A B l1 l2 R D beta n -
    const double *tri;  // (ns^3, 8):   valid c d h l3 m gam -
    double rc;
};

// Per-slot geometry, once per call: d (minimum image), r, the tangent t and
// a live flag (inside the cutoff), 8 doubles per slot.
struct SlotGeo {
    double d[3], r, t[3], live;
};

// live[s] = 1 for a bond that contributes (inside the cutoff, pair record
// valid): the slots the site passes run over, compacted by a scan.
__global__ void te_adjoint_prep(SysView S, const int *__restrict__ row_off, const int *__restrict__ nbr,
                                AdjTab P, AdjIn G, int n_slots, SlotGeo *__restrict__ geo,
                                int *__restrict__ live, int *__restrict__ inside) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_slots) return;
    SlotGeo o;
    o.live = 0.0;
    o.d[0] = o.d[1] = o.d[2] = o.r = o.t[0] = o.t[1] = o.t[2] = 0.0;
    int bond = 0;
    if (s < row_off[S.n_atoms]) {
        int i = slot_owner(row_off, S.n_atoms, s);
        int j = nbr[s];
        int sst = S.n_struct > 1 ? S.atom_struct[i] : 0;
        adj_leg(S, G, cell_of(S, i), i, j, sst, o.d, o.r, o.t);
        o.live = (o.r < P.rc && o.r > 1e-12) ? 1.0 : 0.0;
        if (o.live != 0.0) {
            int si = S.types[i], sj = S.types[j];
            int lo = i < j ? si : sj, hi = i < j ? sj : si;
            bond = P.tb[10 * (lo * P.ns + hi)] != 0.0 ? 1 : 0;
        }
    }
    geo[s] = o;
    live[s] = bond;
    inside[s] = o.live != 0.0 ? 1 : 0;
}

__global__ void te_adjoint_compact(int n_slots, const int *__restrict__ live, const int *__restrict__ pos,
                                   int *__restrict__ bonds) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n_slots && live[s]) bonds[pos[s]] = s;
}

// One zeta term gamma fc(r_ik) g(theta) exp((lambda3 (r_ij - r_ik))^m)
// (engine/tersoff.py:63-101, :528-540) in hyper-dual arithmetic; zero (a
// constant) where fc(r_ik) = 0, as the reference skips it.
template <int K>
__device__ __forceinline__ HD<K> te_zterm(const HD<K> &r, const HD<K> &rk, const HD<K> &dot, const HD<K> &Rk,
                                          const HD<K> &Dk, const HD<K> &c, const HD<K> &d, const HD<K> &h,
                                          const HD<K> &l3, const HD<K> &gam, double m) {
    HD<K> fck = hd_fc<K>(rk, Rk, Dk);
    if (fck.v == 0.0) return hd_const<K>(0.0);
    HD<K> cs = dot / (r * rk);
    HD<K> hc = h - cs;
    HD<K> d2 = d * d, hc2 = hc * hc;
    HD<K> g = 1.0 + ((c * c) * hc2) / (d2 * (d2 + hc2));
    HD<K> ex = hd_cexp<K>(hd_arg<K>(l3, r - rk, m));
    return gam * fck * g * ex;
}

// b(zeta) = (1 + (beta zeta)^n)^(-1/(2n)) for zeta > 0 and beta != 0, else 1
// (engine/tersoff.py:1380-1391).
template <int K>
__device__ __forceinline__ HD<K> te_bond_order(const HD<K> &zeta, const HD<K> &beta, const HD<K> &nn) {
    if (!(zeta.v > 0.0 && beta.v != 0.0)) return hd_const<K>(1.0);
    HD<K> bz = hd_pow<K>(beta * zeta, nn);
    return hd_exp<K>(hd_log<K>(1.0 + bz) * ((-0.5) * hd_inv<K>(nn)));
}

// Every site of one live bond in one pass.  With V = 1/2 fc (fR + b(zeta)
// fA) and Q = gE V + D_t V:
//   the pair and bond-order sites (0..7) from one evaluation of V in
//   hyper-dual arithmetic with zeta held as a (value, tangent) pair;
//   a leg site theta of term k enters only through zeta, so
//   dQ/dtheta = (gE V_z + (V_z)') dz_k/dtheta + V_z d(z_k')/dtheta,
//   V_z = dV/dzeta and (V_z)' its tangent (a dual evaluation), and the
//   term's own derivatives from a hyper-dual over its 7 leg sites.
template <int K>
__device__ int adj_bond_sites(const SysView &S, const int *__restrict__ row_off, const int *__restrict__ nbr,
                              const AdjTab &P, const AdjIn &G, const SlotGeo *__restrict__ geo,
                              const int *__restrict__ legs, const int *__restrict__ lpos, int s, int W,
                              double *__restrict__ out) {
    const int ns = P.ns;
    const SlotGeo gs = geo[s];
    int i = slot_owner(row_off, S.n_atoms, s);
    int j = nbr[s];
    int si = S.types[i], sj = S.types[j];
    int lo = i < j ? si : sj, hi = i < j ? sj : si;
    const double *tp = P.tb + 10 * (lo * ns + hi);
    int code = (si * ns + sj) * 2 + (i < j ? 1 : 0);
    int sst = S.n_struct > 1 ? S.atom_struct[i] : 0;
    const double *dij = gs.d, *tij = gs.t;
    double rij = gs.r, rt = (dij[0] * tij[0] + dij[1] * tij[1] + dij[2] * tij[2]) / rij;
    int beg = row_off[i], end = row_off[i + 1];
    // 1. zeta and its tangent
    HD<1> r1 = hd_const<1>(rij);
    r1.t = rt;
    HD<1> zeta = hd_const<1>(0.0);
    for (int t = lpos[beg]; t < lpos[end]; ++t) {
        int q = legs[t];
        if (q == s) continue;
        const SlotGeo gk = geo[q];
        int sk = S.types[nbr[q]];
        const double *tk = P.tb + 10 * (si * ns + sk);
        const double *t3 = P.tri + 8 * ((si * ns + sj) * ns + sk);
        if (tk[0] == 0.0 || t3[0] == 0.0) continue;
        HD<1> rk = hd_const<1>(gk.r);
        rk.t = (gk.d[0] * gk.t[0] + gk.d[1] * gk.t[1] + gk.d[2] * gk.t[2]) / gk.r;
        HD<1> dot = hd_const<1>(dij[0] * gk.d[0] + dij[1] * gk.d[1] + dij[2] * gk.d[2]);
        dot.t = tij[0] * gk.d[0] + tij[1] * gk.d[1] + tij[2] * gk.d[2] + dij[0] * gk.t[0] + dij[1] * gk.t[1] +
                dij[2] * gk.t[2];
        zeta = zeta + te_zterm<1>(r1, rk, dot, hd_const<1>(tk[5]), hd_const<1>(tk[6]), hd_const<1>(t3[1]),
                                  hd_const<1>(t3[2]), hd_const<1>(t3[3]), hd_const<1>(t3[4]),
                                  hd_const<1>(t3[6]), t3[5]);
    }
    double ge = G.gE ? G.gE[sst] : 0.0;
    const double *tij_rec = P.tb + 10 * (si * ns + sj);
    // 2. pair and bond-order sites
    {
        HD<K> r = hd_const<K>(rij);
        r.t = rt;
        HD<K> z = hd_const<K>(zeta.v);
        z.t = zeta.t;
        HD<K> A = hd_param<K>(tp[1], 0, 0), B = hd_param<K>(tp[2], 1, 0);
        HD<K> l1 = hd_param<K>(tp[3], 2, 0), l2 = hd_param<K>(tp[4], 3, 0);
        HD<K> Rp = hd_param<K>(tp[5], 4, 0), Dp = hd_param<K>(tp[6], 5, 0);
        HD<K> beta = hd_param<K>(tij_rec[7], 6, 0), nn = hd_param<K>(tij_rec[8], 7, 0);
        HD<K> fc = hd_fc<K>(r, Rp, Dp);
        HD<K> fr = A * hd_cexp<K>((-1.0) * (l1 * r));
        HD<K> fa = (-1.0) * (B * hd_cexp<K>((-1.0) * (l2 * r)));
        HD<K> V = 0.5 * (fc * (fr + te_bond_order<K>(z, beta, nn) * fa));
#pragma unroll
        for (int q = 0; q < 8; ++q) out[q] = ge * V.p[q] + V.q[q];
    }
    // 3. V_z = 1/2 fc fA db/dzeta and its tangent
    double c1 = 0.0, c2 = 0.0;
    if (zeta.v > 0.0 && tij_rec[7] != 0.0) {
        HD<1> fc = hd_fc<1>(r1, hd_const<1>(tp[5]), hd_const<1>(tp[6]));
        HD<1> fa = (-tp[2]) * hd_cexp<1>((-tp[4]) * r1);
        HD<1> beta = hd_const<1>(tij_rec[7]), nn = hd_const<1>(tij_rec[8]);
        HD<1> b = te_bond_order<1>(zeta, beta, nn);
        HD<1> u = hd_pow<1>(beta * zeta, nn);
        HD<1> db = (-0.5) * (b * u / (zeta * (1.0 + u)));
        HD<1> Vz = 0.5 * (fc * fa * db);
        c1 = ge * Vz.v + Vz.t;
        c2 = Vz.v;
    }
    // 4. the leg sites of every term, by the species of k
    double acc[8 + 7 * 8];
    for (int w = 8; w < W; ++w) acc[w] = 0.0;
    if (c1 != 0.0 || c2 != 0.0) {
        HD<7> r7 = hd_const<7>(rij);
        r7.t = rt;
        for (int t = lpos[beg]; t < lpos[end]; ++t) {
            int q = legs[t];
            if (q == s) continue;
            const SlotGeo gk = geo[q];
            int sk = S.types[nbr[q]];
            const double *tk = P.tb + 10 * (si * ns + sk);
            const double *t3 = P.tri + 8 * ((si * ns + sj) * ns + sk);
            if (tk[0] == 0.0 || t3[0] == 0.0) continue;
            HD<7> rk = hd_const<7>(gk.r);
            rk.t = (gk.d[0] * gk.t[0] + gk.d[1] * gk.t[1] + gk.d[2] * gk.t[2]) / gk.r;
            HD<7> dot = hd_const<7>(dij[0] * gk.d[0] + dij[1] * gk.d[1] + dij[2] * gk.d[2]);
            dot.t = tij[0] * gk.d[0] + tij[1] * gk.d[1] + tij[2] * gk.d[2] + dij[0] * gk.t[0] + dij[1] * gk.t[1] +
                    dij[2] * gk.t[2];
            HD<7> z = te_zterm<7>(r7, rk, dot, hd_param<7>(tk[5], 5, 0), hd_param<7>(tk[6], 6, 0),
                                  hd_param<7>(t3[1], 0, 0), hd_param<7>(t3[2], 1, 0), hd_param<7>(t3[3], 2, 0),
                                  hd_param<7>(t3[4], 3, 0), hd_param<7>(t3[6], 4, 0), t3[5]);
            double *a = acc + 8 + 7 * sk;
#pragma unroll
            for (int w = 0; w < 7; ++w) a[w] += c1 * z.p[w] + c2 * z.q[w];
        }
    }
    for (int w = 8; w < W; ++w) out[w] = acc[w];
    return code;
}

// Site values of one entry (tb (ns*ns, 10) then tri (ns^3, 8), the tables'
// own layout) summed over `cnt` staged bonds in bond order.
__device__ __forceinline__ double adj_entry_sum(int e, int ns, int W, int cnt, const double *__restrict__ sm,
                                               const int *__restrict__ scode) {
    double a = 0.0;
    if (e < 10 * ns * ns) {
        int row = e / 10, col = e % 10, ra = row / ns, rb = row % ns;
        for (int q = 0; q < cnt; ++q) {
            int c = scode[q];
            if (c < 0) continue;
            int lower = c & 1, pij = c >> 1, si = pij / ns, sj = pij % ns;
            int lo = lower ? si : sj, hi = lower ? sj : si;
            const double *o = sm + (size_t)q * W;
            if (col >= 1 && col <= 6 && lo == ra && hi == rb) a += o[col - 1];
            if ((col == 7 || col == 8) && si == ra && sj == rb) a += o[6 + col - 7];
            if ((col == 5 || col == 6) && si == ra) a += o[8 + 7 * rb + 5 + (col - 5)];
        }
    } else {
        int e3 = e - 10 * ns * ns;
        int row = e3 / 8, col = e3 % 8;
        int ra = row / (ns * ns), rb = (row / ns) % ns, k = row % ns;
        int site = (col >= 1 && col <= 4) ? col - 1 : (col == 6 ? 4 : -1);
        if (site >= 0) {
            for (int q = 0; q < cnt; ++q) {
                int c = scode[q];
                if (c < 0) continue;
                int pij = c >> 1, si = pij / ns, sj = pij % ns;
                if (si == ra && sj == rb) a += sm[(size_t)q * W + 8 + 7 * k + site];
            }
        }
    }
    return a;
}

// Block b takes live bonds b*ADJ_BLOCK ..: every thread one bond, its site
// values staged in shared memory, then the block's sum of every table entry
// (one thread per entry, bond order) to partial[b].
template <int K>
__global__ void __launch_bounds__(ADJ_BLOCK) te_adjoint_bonds(SysView S, const int *__restrict__ row_off,
                                                              const int *__restrict__ nbr, AdjTab P, AdjIn G,
                                                              const SlotGeo *__restrict__ geo,
                                                              const int *__restrict__ legs,
                                                              const int *__restrict__ lpos,
                                                              const int *__restrict__ bonds,
                                                              const int *__restrict__ n_bonds, int W,
                                                              double *__restrict__ partial) {
    extern __shared__ double sm[];  // ADJ_BLOCK * W site values, then ADJ_BLOCK codes
    int *scode = reinterpret_cast<int *>(sm + (size_t)ADJ_BLOCK * W);
    int nb = *n_bonds;
    int m0 = blockIdx.x * ADJ_BLOCK;
    if (m0 >= nb) return;  // the whole block leaves together
    int m = m0 + threadIdx.x;
    double *out = sm + (size_t)threadIdx.x * W;
    int c = -1;
    if (m < nb) c = adj_bond_sites<K>(S, row_off, nbr, P, G, geo, legs, lpos, bonds[m], W, out);
    scode[threadIdx.x] = c;
    __syncthreads();
    int cnt = min(ADJ_BLOCK, nb - m0);
    int ne = 10 * P.ns * P.ns + 8 * P.ns * P.ns * P.ns;
    for (int e = threadIdx.x; e < ne; e += blockDim.x)
        partial[(size_t)blockIdx.x * ne + e] = adj_entry_sum(e, P.ns, W, cnt, sm, scode);
}


// One warp per entry: lanes take every 32nd block partial, then a fixed
// shuffle tree.
__global__ void te_adjoint_final(const int *__restrict__ n_bonds, int ns, const double *__restrict__ partial,
                                 double *__restrict__ d_tb, double *__restrict__ d_tri) {
    int ne = 10 * ns * ns + 8 * ns * ns * ns;
    int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
    if (e >= ne) return;  // whole warps leave together
    int n_blocks = (*n_bonds + ADJ_BLOCK - 1) / ADJ_BLOCK;
    double acc = 0.0;
    for (int b = l; b < n_blocks; b += 32) acc += partial[(size_t)b * ne + e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MBF_FULL, acc, o);
    if (l == 0) {
        if (e < 10 * ns * ns) d_tb[e] = acc;
        else d_tri[e - 10 * ns * ns] = acc;
    }
}

struct AdjLayout {
    size_t partial, geo, live, pos, bonds, inside, lpos, legs, scan, total;
    int W, ne, n_blocks;
};

static AdjLayout adj_layout(long long n_slots, int ns) {
    AdjLayout L;
    L.W = 8 + 7 * ns;
    L.ne = 10 * ns * ns + 8 * ns * ns * ns;
    L.n_blocks = (int)((n_slots + ADJ_BLOCK - 1) / ADJ_BLOCK);  // at most one block per live-bond tile
    if (L.n_blocks < 1) L.n_blocks = 1;
    size_t o = 0;
    L.partial = o;
    o = align256(o + sizeof(double) * (size_t)L.n_blocks * L.ne);
    L.geo = o;
    o = align256(o + sizeof(SlotGeo) * (size_t)(n_slots > 0 ? n_slots : 1));
    L.live = o;
    o = align256(o + sizeof(int) * (size_t)(n_slots > 0 ? n_slots : 1));
    L.pos = o;
    o = align256(o + sizeof(int) * (size_t)(n_slots + 1));
    L.bonds = o;
    o = align256(o + sizeof(int) * (size_t)(n_slots > 0 ? n_slots : 1));
    L.inside = o;
    o = align256(o + sizeof(int) * (size_t)(n_slots > 0 ? n_slots : 1));
    L.lpos = o;
    o = align256(o + sizeof(int) * (size_t)(n_slots + 1));
    L.legs = o;
    o = align256(o + sizeof(int) * (size_t)(n_slots > 0 ? n_slots : 1));
    L.scan = o;
    o = align256(o + sizeof(int) * scan_workspace_ints((int)(n_slots > 0 ? n_slots : 1)));
    L.total = o;
    return L;
}

}  // namespace mbf

using namespace mbf;

extern "C" {

size_t mbf_tersoff_adjoint_workspace_bytes(long long n_slots, int ns) {
    if (ns <= 0 || n_slots < 0) return 0;
    return adj_layout(n_slots, ns).total;
}

int mbf_tersoff_adjoint(const mbf_system *sys, const mbf_nlist *nl, const mbf_tersoff_tables *tab,
                        const double *g_energy, const double *g_forces, const double *g_virial, void *workspace,
                        size_t workspace_bytes, double *d_tb, double *d_tri, void *stream) {
    if (!sys || !nl || !tab || !workspace || !d_tb || !d_tri || tab->ns <= 0 || tab->ns > 8)
        return MBF_ERR_ARGUMENT;
    if (nl->n_atoms != sys->n_atoms) return MBF_ERR_ARGUMENT;
    AdjLayout L = adj_layout(nl->n_slots, tab->ns);
    if (workspace_bytes < L.total) return MBF_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    int ns = tab->ns;
    if (sys->n_atoms == 0 || nl->n_slots == 0) {
        if (cudaMemsetAsync(d_tb, 0, sizeof(double) * 10 * ns * ns, st) != cudaSuccess ||
            cudaMemsetAsync(d_tri, 0, sizeof(double) * 8 * ns * ns * ns, st) != cudaSuccess)
            return MBF_ERR_CUDA;
        return MBF_OK;
    }
    SysView S = make_view(sys);
    AdjTab P;
    P.ns = ns;
    P.tb = tab->tb;
    P.tri = tab->tri;
    P.rc = tab->r_cut;
    AdjIn G;
    G.gE = g_energy;
    G.gF = g_forces;
    G.gW = g_virial;
    double *partial = ws_at<double>(workspace, L.partial);
    int n_slots = (int)nl->n_slots;
    SlotGeo *geo = ws_at<SlotGeo>(workspace, L.geo);
    int *live = ws_at<int>(workspace, L.live);
    int *pos = ws_at<int>(workspace, L.pos);
    int *bonds = ws_at<int>(workspace, L.bonds);
    int *inside = ws_at<int>(workspace, L.inside);
    int *lpos = ws_at<int>(workspace, L.lpos);
    int *legs = ws_at<int>(workspace, L.legs);
    int grid = (n_slots + ADJ_BLOCK - 1) / ADJ_BLOCK;
    PROF_BEGIN("te_adjoint_prep", st);
    te_adjoint_prep<<<grid, ADJ_BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, P, G, n_slots, geo, live, inside);
    MBF_CHECK_LAUNCH();
    int rc = exclusive_scan(live, pos, n_slots, ws_at<int>(workspace, L.scan), st);
    if (rc != MBF_OK) return rc;
    te_adjoint_compact<<<grid, ADJ_BLOCK, 0, st>>>(n_slots, live, pos, bonds);
    // the slots inside the cutoff, each row's contiguous and in slot order: the
    // zeta loops of a bond run over these only
    rc = exclusive_scan(inside, lpos, n_slots, ws_at<int>(workspace, L.scan), st);
    if (rc != MBF_OK) return rc;
    te_adjoint_compact<<<grid, ADJ_BLOCK, 0, st>>>(n_slots, inside, lpos, legs);
    PROF_END("te_adjoint_prep", st);
    const int *n_bonds = pos + n_slots;  // the scan's total
    size_t smem = (size_t)ADJ_BLOCK * L.W * sizeof(double) + ADJ_BLOCK * sizeof(int);  // <= 33 KB (ns <= 8)
    int bgrid = L.n_blocks;
    PROF_BEGIN("te_adjoint_bonds", st);
    te_adjoint_bonds<ADJ_K><<<bgrid, ADJ_BLOCK, smem, st>>>(S, nl->row_off, nl->nbr, P, G, geo, legs, lpos, bonds,
                                                              n_bonds, L.W, partial);
    PROF_END("te_adjoint_bonds", st);
    MBF_CHECK_LAUNCH();
    PROF_BEGIN("te_adjoint_reduce", st);
    te_adjoint_final<<<(L.ne * 32 + 127) / 128, 128, 0, st>>>(n_bonds, ns, partial, d_tb, d_tri);
    PROF_END("te_adjoint_reduce", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

}  // extern "C"
