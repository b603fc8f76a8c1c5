// Zhou EAM adjoint: the vector-Jacobian product of (E, F, virial) with
// respect to the function rows P (nf, 43) of an analytic Zhou (2004) table,
// for fitting.
//
// As for the Tersoff adjoint, the pull-back of upstream gradients gE, gF, gW
// onto a parameter theta is d/dtheta [sum_s gE_s E_s + D_t E], D_t the
// derivative along the tangent field t_ij = gF_i - gF_j - gW d_ij of the pair
// vectors.  The energy is a sum of site terms
//
//   U_i = F_{s_i}(rho-bar_i) + 1/2 sum_j phi_{s_i s_j}(r_ij),
//   rho-bar_i = sum_j rho_{s_j}(r_ij)      (engine/eam.py:174-256),
//
// with the Zhou forms of engine/eam_zhou.py:20-115 (density and pair
// functions times the quintic switch, the cross pair
// 1/2 k (f_b/f_a phi_aa + f_a/f_b phi_bb), embedding eqs. (A6)-(A8)).
// Per atom, in float64 hyper-dual arithmetic (one tangent, K parameter
// directions):
//   Q_i = gE F(rho-bar) + F'(rho-bar) D_t rho-bar + 1/2 sum_j (gE phi + D_t phi).
// The embedding's 12 parameters and rho-bar itself are the 13 directions of
// one evaluation of F; with c1 = gE F' + F'' D_t rho-bar and c2 = F', a
// density parameter's site value is c1 d(rho)/dtheta + c2 d(D_t rho)/dtheta.
// Density and pair functions are built from decays
// g(r; r_e, exponent, shift), each differentiated in its own three
// parameters only; an element's eight parameters and the cross pair's
// (f_a, u_a, f_b, u_b) dependence are chained by hand from those.
//
// Sites of atom i (W = 12 + 21 ns):
//   0..11               rho_e, rho_s, Fn0..Fn3, F0..F3, eta, F_e of row F_f[s_i]
//                       (columns 2, 3, 10..19)
//   12 + 4 s + 0..3     r_e, f_e, beta, lambda of row rho_f[s] (columns 0, 1, 5, 9)
//   12 + 4 ns + 17 s    the pair row phi_f[s_i, s]: 0..7 the earlier species'
//                       r_e, f_e, alpha, beta, A, B, kappa, lambda (columns 0,
//                       1, 4..9), 8..15 the later species' (columns 20, 21,
//                       24..29, cross rows only), 16 the factor k (column 42)
// Columns 40, 41 (switch radius and width) are not differentiated: the
// cutoff is fixed during a fit.  The gradient is with respect to the rows
// the generic Zhou evaluation reads (rho_f, F_f, phi_f); the fused path
// reads the same element parameters from the density rows, which the table
// builders fill identically.  Sites are reduced onto the entries in a fixed
// order: deterministic.
#include "mbf_hd.cuh"

namespace mbf {

constexpr int EADJ_NCOL = 43;
constexpr int EADJ_NZ = 20;

struct EamAdjTab {
    int ns, nf;
    const double *P;
    const int *rho_f, *F_f, *phi_f;
    double rc;
};

// g = exp(-expo (x - 1)) / (1 + (x - shift)^20), x = r / re, the decay
// every Zhou function is built from (engine/eam_zhou.py:20-45), with r's
// tangent rt; as HD<3> its directions are (re, expo, shift).
template <int K>
__device__ __forceinline__ HD<K> hz_decay(double r, double rt, const HD<K> &re, const HD<K> &expo,
                                          const HD<K> &shift) {
    HD<K> R = hd_const<K>(r);
    R.t = rt;
    HD<K> x = R / re;
    HD<K> e = hd_exp<K>((-1.0) * (expo * (x + (-1.0))));
    HD<K> u = x - shift;
    double u2 = u.v * u.v, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8, u18 = u16 * u2;
    HD<K> den = 1.0 + hd_apply<K>(u, u18 * u2, 20.0 * u18 * u.v, 380.0 * u18);
    return e / den;
}

__device__ __forceinline__ HD<3> hz_g3(double r, double rt, double re, double expo, double shift) {
    return hz_decay<3>(r, rt, hd_param<3>(re, 0, 0), hd_param<3>(expo, 1, 0), hd_param<3>(shift, 2, 0));
}

// The quintic switch of a row (columns 40, 41) at r: value and tangent.
__device__ __forceinline__ void hz_switch(const double *row, double r, double rt, double &S, double &St) {
    double rc = row[2 * EADJ_NZ], w = row[2 * EADJ_NZ + 1];
    double s = (r - (rc - w)) / w;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
    S = 1.0 - s * s * s * (10.0 - 15.0 * s + 6.0 * s * s);
    St = -30.0 * s * s * (1.0 - s) * (1.0 - s) / w * rt;
}

// One element's density f = f_e gB and pair u = A gA - B gB (unswitched),
// gA = g(r; r_e, alpha, kappa), gB = g(r; r_e, beta, lambda), enter a site
// value through their parameter derivatives (p) and the tangent of those
// (q): site_k += af f.p_k + bf f.q_k + au u.p_k + bu u.q_k, for the 8
// element parameters r_e, f_e, alpha, beta, A, B, kappa, lambda (columns 0,
// 1, 4..9 of p).
__device__ __forceinline__ void hz_species_sites(double *o, const HD<3> &gA, const HD<3> &gB, const double *p,
                                                 double af, double bf, double au, double bu) {
    double fe = p[1], A = p[6], B = p[7];
    o[0] += fe * (af * gB.p[0] + bf * gB.q[0]) + au * (A * gA.p[0] - B * gB.p[0]) + bu * (A * gA.q[0] - B * gB.q[0]);
    o[1] += af * gB.v + bf * gB.t;
    o[2] += A * (au * gA.p[1] + bu * gA.q[1]);
    o[3] += (fe * af - B * au) * gB.p[1] + (fe * bf - B * bu) * gB.q[1];
    o[4] += au * gA.v + bu * gA.t;
    o[5] -= au * gB.v + bu * gB.t;
    o[6] += A * (au * gA.p[2] + bu * gA.q[2]);
    o[7] += (fe * af - B * au) * gB.p[2] + (fe * bf - B * bu) * gB.q[2];
}

// Zhou embedding F(rho), eqs. (A6)-(A8) (engine/eam_zhou.py:66-115), with
// rho_e, rho_s, Fn0..3, F0..3, eta, F_e (columns 2, 3, 10..19) as directions
// 0..11 and rho itself as direction 12.
__device__ __forceinline__ HD<13> hz_embed(const double *p, double rho, double rho_t) {
    HD<13> q[12];
    const int col[12] = {2, 3, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19};
#pragma unroll
    for (int k = 0; k < 12; ++k) q[k] = hd_param<13>(p[col[k]], k, 0);
    HD<13> x = hd_param<13>(rho, 12, 0);
    x.t = rho_t;
    const HD<13> &re = q[0], &rs = q[1], &eta = q[10], &Fe = q[11];
    if (rho < 0.85 * re.v) {
        HD<13> z = x / (0.85 * re) + (-1.0);
        return q[2] + z * (q[3] + z * (q[4] + z * q[5]));
    }
    if (rho >= 1.15 * re.v) {
        HD<13> lt = hd_log<13>(x / rs);
        HD<13> el = eta * lt;
        return Fe * ((1.0 + (-1.0) * el) * hd_exp<13>(el));
    }
    HD<13> z = x / re + (-1.0);
    return q[6] + z * (q[7] + z * (q[8] + z * q[9]));
}

__device__ __forceinline__ const double *row_of(const EamAdjTab &T, int f) { return T.P + (size_t)f * EADJ_NCOL; }

// Value and r-tangent of f_e g(r; r_e, beta, lambda) S(r) for pass 1.
__device__ __forceinline__ void dens_value(const double *row, double r, double rt, double &v, double &vt) {
    double x = r / row[0];
    double e = exp(-row[5] * (x - 1.0));
    double u = x - row[9];
    double u2 = u * u, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8, u19 = u16 * u2 * u;
    double id = 1.0 / (1.0 + u19 * u);
    double g = e * id;
    double dg = g * (-row[5] - 20.0 * u19 * id) / row[0];
    double Sw, St;
    hz_switch(row, r, 1.0, Sw, St);  // St = dS/dr here
    v = row[1] * g * Sw;
    vt = row[1] * (dg * Sw + g * St) * rt;
}

// Tiles: EADJ_TA atoms (embedding pass) or EADJ_TP pairs (pair pass) per
// iteration of a block; blocks stride over tiles in a fixed order and keep
// their own sums, so every reduction below is in a fixed order.
constexpr int EADJ_TA = 128;
constexpr int EADJ_TP = 64;
constexpr int EADJ_GRID = 148 * 16;  // pair-kernel blocks at most (16 per SM of a B200)
constexpr int EADJ_PS = 25;          // staged values of one pair
constexpr int EADJ_STRIDE = 25;      // odd: conflict-free 8-byte shared accesses

// Pass 1, a thread per atom: rho-bar and its tangent over the full row, the
// embedding sites (12; summed per species of the centre into the block's
// partialF row) and the coefficients c1 = gE F' + F'' D_t rho-bar, c2 = F'
// through which every density parameter acts on this atom's site term.
// Also counts the live pairs above the diagonal (j > i, inside the cutoff):
// cnt[i] like-species pairs, cnt[n_atoms + i] cross pairs.
__global__ void __launch_bounds__(EADJ_TA) eam_adjoint_embed(SysView S, const int *__restrict__ row_off,
                                                             const int *__restrict__ upper,
                                                             const int *__restrict__ nbr, EamAdjTab T, AdjIn G,
                                                             double2 *__restrict__ cc, int *__restrict__ cnt,
                                                             double *__restrict__ partialF) {
    __shared__ double sf[EADJ_TA * 13];  // 12 sites per atom, odd stride
    __shared__ int scode[EADJ_TA];
    extern __shared__ double accF[];     // ns * 12
    const int ns = T.ns, nf = 12 * ns;
    for (int k = threadIdx.x; k < nf; k += blockDim.x) accF[k] = 0.0;
    const double rc2 = T.rc * T.rc;
    int n_tiles = (S.n_atoms + EADJ_TA - 1) / EADJ_TA;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        int i = tile * EADJ_TA + threadIdx.x;
        int code = -1;
        double *o = sf + 13 * threadIdx.x;
        if (i < S.n_atoms) {
            int si = S.types[i];
            int sst = S.n_struct > 1 ? S.atom_struct[i] : 0;
            double gE = G.gE ? G.gE[sst] : 0.0;
            const double *cell = cell_of(S, i);
            double rho = 0.0, rho_t = 0.0;
            int up = upper[i], n_like = 0, n_cross = 0;
            for (int s = row_off[i]; s < row_off[i + 1]; ++s) {
                int j = nbr[s];
                double d[3], r, tg[3];
                adj_leg(S, G, cell, i, j, sst, d, r, tg);
                if (!(r * r < rc2 && r * r > 1e-24)) continue;
                int sj = S.types[j];
                if (s >= up) {
                    if (si == sj) ++n_like;
                    else ++n_cross;
                }
                double rt = (d[0] * tg[0] + d[1] * tg[1] + d[2] * tg[2]) / r;
                double v, vt;
                dens_value(row_of(T, T.rho_f[sj]), r, rt, v, vt);
                rho += v;
                rho_t += vt;
            }
            // the embedding, rho-bar clamped at 0 as the evaluation does
            double rb = rho > 0.0 ? rho : 0.0;
            HD<13> F = hz_embed(row_of(T, T.F_f[si]), rb, rho_t);
#pragma unroll
            for (int k = 0; k < 12; ++k) o[k] = gE * F.p[k] + F.q[k];
            cc[i] = make_double2(rho > 0.0 ? gE * F.p[12] + F.q[12] : 0.0, F.p[12]);
            cnt[i] = n_like;
            cnt[S.n_atoms + i] = n_cross;
            code = si;
        }
        scode[threadIdx.x] = code;
        __syncthreads();
        int cnt = min(EADJ_TA, S.n_atoms - tile * EADJ_TA);
        for (int item = threadIdx.x; item < nf; item += blockDim.x) {
            int sp = item / 12, k = item % 12;
            double a = 0.0;
            for (int q = 0; q < cnt; ++q)
                if (scode[q] == sp) a += sf[13 * q + k];
            accF[item] += a;
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < nf; k += blockDim.x) partialF[(size_t)blockIdx.x * nf + k] = accF[k];
}

// Compacted pair list, a thread per atom: its live upper slots (the same
// test as eam_adjoint_embed's, so the same count) at its scanned offsets,
// like pairs in [pos[0], pos[N]), cross pairs in [pos[N], pos[2N]), each in
// atom then slot order.
__global__ void eam_adjoint_compact(SysView S, const int *__restrict__ row_off, const int *__restrict__ upper,
                                    const int *__restrict__ nbr, EamAdjTab T, AdjIn G,
                                    const int *__restrict__ pos, int *__restrict__ pairs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n_atoms) return;
    int si = S.types[i];
    int sst = S.n_struct > 1 ? S.atom_struct[i] : 0;
    const double *cell = cell_of(S, i);
    const double rc2 = T.rc * T.rc;
    int ol = pos[i], oc = pos[S.n_atoms + i];
    for (int s = upper[i]; s < row_off[i + 1]; ++s) {
        int j = nbr[s];
        double d[3], r, tg[3];
        adj_leg(S, G, cell, i, j, sst, d, r, tg);
        if (!(r * r < rc2 && r * r > 1e-24)) continue;
        if (S.types[j] == si) pairs[ol++] = s;
        else pairs[oc++] = s;
    }
}

// The slot's owning atom: rows are sorted, so a binary search in row_off.
__device__ __forceinline__ int eadj_owner(const int *__restrict__ row_off, int n_atoms, int s) {
    int lo = 0, hi = n_atoms - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (row_off[mid] <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Density sites of one centre's view of a neighbour of species s at r:
// rho_s = f_e gB S, contributing c1 d(rho)/dtheta + c2 d(D_t rho)/dtheta to
// r_e, f_e, beta, lambda (o[0..3]).
__device__ __forceinline__ void dens_sites(double *o, const HD<3> &gB, const double *row, double Sw, double St,
                                           double c1, double c2) {
    double a = c1 * Sw + c2 * St, bq = c2 * Sw;
    double af = a * row[1], bf = bq * row[1];
    o[0] += af * gB.p[0] + bf * gB.q[0];
    o[1] += a * gB.v + bq * gB.t;
    o[2] += af * gB.p[1] + bf * gB.q[1];
    o[3] += af * gB.p[2] + bf * gB.q[2];
}

// The density decay of species row `dr` at r: the pair's decay of the same
// element when the density row holds the same (r_e, beta, lambda), else its
// own.
__device__ __forceinline__ HD<3> dens_decay(const double *dr, const double *blk, const HD<3> &gB_blk, double r,
                                            double rt) {
    if (dr[0] == blk[0] && dr[5] == blk[5] && dr[9] == blk[9]) return gB_blk;
    return hz_g3(r, rt, dr[0], dr[5], dr[9]);
}

// The 25 staged values of the live pair at slot s (i < j): 0..16 the pair
// sites of row phi_f[s_i, s_j] (weight 1: the two halves 1/2 phi of the
// site terms of i and j), 17..20 the density sites of i's view of rho_{s_j}
// (coefficients of i), 21..24 those of j's view of rho_{s_i}.  Returns the
// code s_i ns + s_j.
template <bool LIKE>
__device__ int eam_pair_sites(const SysView &S, const int *__restrict__ row_off, const int *__restrict__ nbr,
                              const EamAdjTab &T, const AdjIn &G, const double2 *__restrict__ cc, int s, double *o) {
    const int ns = T.ns;
    int i = eadj_owner(row_off, S.n_atoms, s);
    int j = nbr[s];
    int si = S.types[i], sj = S.types[j];
    int sst = S.n_struct > 1 ? S.atom_struct[i] : 0;
    double gE = G.gE ? G.gE[sst] : 0.0;
    double d[3], r, tg[3];
    adj_leg(S, G, cell_of(S, i), i, j, sst, d, r, tg);
    double rt = (d[0] * tg[0] + d[1] * tg[1] + d[2] * tg[2]) / r;
    for (int k = 0; k < EADJ_PS; ++k) o[k] = 0.0;
    const double *row = row_of(T, T.phi_f[si * ns + sj]);
    const double *rho_i = row_of(T, T.rho_f[si]), *rho_j = row_of(T, T.rho_f[sj]);
    const double2 ci = cc[i], cj = cc[j];
    double Sw, St, Dw, Dt;
    hz_switch(row, r, rt, Sw, St);
    HD<3> gAa = hz_g3(r, rt, row[0], row[4], row[8]);
    HD<3> gBa = hz_g3(r, rt, row[0], row[5], row[9]);
    if (LIKE) {
        // phi = u S
        hz_species_sites(o, gAa, gBa, row, 0.0, 0.0, gE * Sw + St, Sw);
        HD<3> gD = dens_decay(rho_j, row, gBa, r, rt);
        hz_switch(rho_j, r, rt, Dw, Dt);
        dens_sites(o + 17, gD, rho_j, Dw, Dt, ci.x, ci.y);
        dens_sites(o + 21, gD, rho_i, Dw, Dt, cj.x, cj.y);
    } else {
        // phi = k psi, psi = 1/2 S (q u_a + u_b / q), q = f_b / f_a, a the
        // earlier species: psi's derivatives in (f_a, u_a, f_b, u_b), then
        // each element's chain
        const double *pb = row + EADJ_NZ;
        HD<3> gAb = hz_g3(r, rt, pb[0], pb[4], pb[8]);
        HD<3> gBb = hz_g3(r, rt, pb[0], pb[5], pb[9]);
        HD<4> fa = hd_param<4>(row[1] * gBa.v, 0, 0), ua = hd_param<4>(row[6] * gAa.v - row[7] * gBa.v, 1, 0);
        HD<4> fb = hd_param<4>(pb[1] * gBb.v, 2, 0), ub = hd_param<4>(pb[6] * gAb.v - pb[7] * gBb.v, 3, 0);
        fa.t = row[1] * gBa.t;
        ua.t = row[6] * gAa.t - row[7] * gBa.t;
        fb.t = pb[1] * gBb.t;
        ub.t = pb[6] * gAb.t - pb[7] * gBb.t;
        HD<4> Sh = hd_const<4>(Sw);
        Sh.t = St;
        HD<4> q = fb / fa;
        HD<4> psi = 0.5 * (Sh * (q * ua + ub / q));
        double h = row[2 * EADJ_NZ + 2];
        hz_species_sites(o, gAa, gBa, row, h * (gE * psi.p[0] + psi.q[0]), h * psi.p[0],
                         h * (gE * psi.p[1] + psi.q[1]), h * psi.p[1]);
        hz_species_sites(o + 8, gAb, gBb, pb, h * (gE * psi.p[2] + psi.q[2]), h * psi.p[2],
                         h * (gE * psi.p[3] + psi.q[3]), h * psi.p[3]);
        o[16] = gE * psi.v + psi.t;
        // the element blocks of s_i and s_j in the cross row
        bool i_first = si < sj;
        const double *bi = i_first ? row : pb, *bj = i_first ? pb : row;
        HD<3> gDj = dens_decay(rho_j, bj, i_first ? gBb : gBa, r, rt);
        hz_switch(rho_j, r, rt, Dw, Dt);
        dens_sites(o + 17, gDj, rho_j, Dw, Dt, ci.x, ci.y);
        HD<3> gDi = dens_decay(rho_i, bi, i_first ? gBa : gBb, r, rt);
        hz_switch(rho_i, r, rt, Dw, Dt);
        dens_sites(o + 21, gDi, rho_i, Dw, Dt, cj.x, cj.y);
    }
    return si * ns + sj;
}

// Pass 2, a thread per live pair of one segment of the compacted list
// (like pairs [0, pos[N]) or cross pairs [pos[N], pos[2 N])), EADJ_TP
// pairs per tile: the staged values are sorted by code
// inside the tile (a counting sort, ranks from warp matches, so the order
// is fixed), then each (code, value) item is summed over its segment into
// the block's partialP row (ns^2 * 25).  The two segments are separate
// instantiations: the like pairs' kernel keeps a smaller register budget.
// Resident blocks per SM the cross-pair instantiation is compiled for (its
// register budget: 65536 / (EADJ_TP * MBF_EADJ_CROSS_MINB)).
#ifndef MBF_EADJ_CROSS_MINB
#define MBF_EADJ_CROSS_MINB 8
#endif

template <bool LIKE>
__global__ void __launch_bounds__(EADJ_TP, LIKE ? 1 : MBF_EADJ_CROSS_MINB) eam_adjoint_pairs(SysView S, const int *__restrict__ row_off,
                                                             const int *__restrict__ nbr, EamAdjTab T, AdjIn G,
                                                             const double2 *__restrict__ cc,
                                                             const int *__restrict__ pairs,
                                                             const int *__restrict__ seg_begin,
                                                             const int *__restrict__ seg_end,
                                                             double *__restrict__ partialP) {
    __shared__ double st[EADJ_TP * EADJ_STRIDE];
    __shared__ int order[EADJ_TP];
    __shared__ int wcnt[2][65], start[66];
    extern __shared__ double accP[];     // ns^2 * 25
    const int ns = T.ns, nc = ns * ns, ni = nc * EADJ_PS;
    for (int k = threadIdx.x; k < ni; k += blockDim.x) accP[k] = 0.0;
    const int p0 = *seg_begin, np = *seg_end - p0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int tile = blockIdx.x; tile * EADJ_TP < np; tile += gridDim.x) {
        int m = tile * EADJ_TP + threadIdx.x;
        int code = nc;  // past the last code: not summed
        if (m < np)
            code = eam_pair_sites<LIKE>(S, row_off, nbr, T, G, cc, pairs[p0 + m], st + EADJ_STRIDE * threadIdx.x);
        for (int k = threadIdx.x; k < 2 * 65; k += blockDim.x) (&wcnt[0][0])[k] = 0;
        __syncthreads();
        unsigned same = __match_any_sync(MBF_FULL, code);
        int rank = __popc(same & ((1u << lane) - 1u));
        if (rank == 0) wcnt[w][code] = __popc(same);
        __syncthreads();
        if (threadIdx.x == 0) {
            int a = 0;
            for (int c = 0; c <= nc; ++c) {
                start[c] = a;
                a += wcnt[0][c] + wcnt[1][c];
            }
            start[nc + 1] = a;
        }
        __syncthreads();
        order[start[code] + (w ? wcnt[0][code] : 0) + rank] = threadIdx.x;
        __syncthreads();
        for (int item = threadIdx.x; item < ni; item += blockDim.x) {
            int c = item / EADJ_PS, k = item % EADJ_PS;
            double a = 0.0;
            for (int q = start[c]; q < start[c + 1]; ++q) a += st[EADJ_STRIDE * order[q] + k];
            accP[item] += a;
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < ni; k += blockDim.x) partialP[(size_t)blockIdx.x * ni + k] = accP[k];
}

// Column -> site of a role (-1: not differentiated).
__device__ __forceinline__ int f_site(int c) { return c == 2 ? 0 : (c == 3 ? 1 : (c >= 10 && c <= 19 ? c - 8 : -1)); }
__device__ __forceinline__ int d_site(int c) { return c == 0 ? 0 : (c == 1 ? 1 : (c == 5 ? 2 : (c == 9 ? 3 : -1))); }
__device__ __forceinline__ int p_site(int c) {
    if (c == 0 || c == 1) return c;
    if (c >= 4 && c <= 9) return c - 2;
    if (c == 20 || c == 21) return c - 12;
    if (c >= 24 && c <= 29) return c - 14;
    return c == 42 ? 16 : -1;
}

// One warp per entry (row f, column c) of d_P: the block partials that feed
// it -- the embedding sums of the row's species, the density values of
// every code with that neighbour (i's view) or centre (j's view) species,
// the pair values of the row's code(s) -- summed over blocks by lanes, then
// a fixed shuffle tree.
__global__ void eam_adjoint_final(EamAdjTab T, int gA, const double *__restrict__ partialF, int gP,
                                  const double *__restrict__ partialP, double *__restrict__ d_P) {
    const int ns = T.ns, nfs = 12 * ns, ni = ns * ns * EADJ_PS;
    int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
    if (e >= T.nf * EADJ_NCOL) return;  // whole warps leave together
    int f = e / EADJ_NCOL, c = e % EADJ_NCOL;
    int idx[16], n = 0;  // items of partialP feeding this entry (<= 2 ns)
    int fitem = -1;      // item of partialF
    for (int s = 0; s < ns; ++s) {
        if (T.F_f[s] == f && f_site(c) >= 0) fitem = 12 * s + f_site(c);
        if (T.rho_f[s] == f && d_site(c) >= 0)
            for (int x = 0; x < ns; ++x) {
                idx[n++] = (x * ns + s) * EADJ_PS + 17 + d_site(c);  // centre x, neighbour s
                idx[n++] = (s * ns + x) * EADJ_PS + 21 + d_site(c);  // centre s: j's view
            }
    }
    for (int x = 0; x < ns; ++x)
        for (int y = x; y < ns; ++y) {
            int k = p_site(c);
            if (T.phi_f[x * ns + y] != f || k < 0 || (x == y && k >= 8)) continue;
            idx[n++] = (x * ns + y) * EADJ_PS + k;
            if (x != y) idx[n++] = (y * ns + x) * EADJ_PS + k;
        }
    double acc = 0.0;
    if (fitem >= 0)
        for (int b = l; b < gA; b += 32) acc += partialF[(size_t)b * nfs + fitem];
    for (int b = l; b < gP; b += 32) {  // the like and the cross kernels' rows
        const double *pp = partialP + (size_t)b * ni;
        for (int q = 0; q < n; ++q) acc += pp[idx[q]];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MBF_FULL, acc, o);
    if (l == 0) d_P[e] = acc;
}

// Workspace of one call.
struct EadjLayout {
    size_t partialF, partialP, cc, cnt, pos, pairs, scan, total;
    int gA, gP;
};

static EadjLayout eadj_layout(int n_atoms, long long n_slots, int ns) {
    EadjLayout L;
    long long ns2 = n_slots > 0 ? n_slots : 1;
    int tiles_a = (int)((n_atoms + EADJ_TA - 1) / EADJ_TA);
    long long tiles_p = (ns2 + EADJ_TP - 1) / EADJ_TP;  // the live pairs are at most the slots
    L.gA = tiles_a < 1 ? 1 : (tiles_a < 65535 ? tiles_a : 65535);
    L.gP = (int)(tiles_p < EADJ_GRID ? tiles_p : EADJ_GRID);  // rows per pair kernel, at most
    if (L.gP < 1) L.gP = 1;
    size_t o = 0;
    L.partialF = o;
    o = align256(o + sizeof(double) * (size_t)L.gA * 12 * ns);
    L.partialP = o;
    o = align256(o + sizeof(double) * (size_t)2 * L.gP * ns * ns * EADJ_PS);
    L.cc = o;
    o = align256(o + sizeof(double2) * (size_t)(n_atoms > 0 ? n_atoms : 1));
    size_t na = (size_t)(n_atoms > 0 ? n_atoms : 1);
    L.cnt = o;
    o = align256(o + sizeof(int) * 2 * na);
    L.pos = o;
    o = align256(o + sizeof(int) * (2 * na + 1));
    L.pairs = o;
    o = align256(o + sizeof(int) * (size_t)ns2);
    L.scan = o;
    o = align256(o + sizeof(int) * scan_workspace_ints((int)(2 * na)));
    L.total = o;
    return L;
}

}  // namespace mbf

using namespace mbf;

extern "C" {

size_t mbf_eam_adjoint_workspace_bytes(int n_atoms, long long n_slots, int ns) {
    if (n_atoms < 0 || n_slots < 0 || ns <= 0 || ns > 8 || n_slots > 0x7fffffffLL) return 0;
    return eadj_layout(n_atoms, n_slots, ns).total;
}

int mbf_eam_adjoint(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab, const double *g_energy,
                    const double *g_forces, const double *g_virial, void *workspace, size_t workspace_bytes,
                    double *d_P, void *stream) {
    if (!sys || !nl || !tab || !workspace || !d_P || tab->ns <= 0 || tab->ns > 8 || tab->nf <= 0)
        return MBF_ERR_ARGUMENT;
    if (nl->n_atoms != sys->n_atoms || !nl->upper || nl->n_slots > 0x7fffffffLL) return MBF_ERR_ARGUMENT;
    EadjLayout L = eadj_layout(sys->n_atoms, nl->n_slots, tab->ns);
    if (workspace_bytes < L.total) return MBF_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    int ne = tab->nf * EADJ_NCOL;
    if (sys->n_atoms == 0) {
        if (cudaMemsetAsync(d_P, 0, sizeof(double) * ne, st) != cudaSuccess) return MBF_ERR_CUDA;
        return MBF_OK;
    }
    SysView S = make_view(sys);
    EamAdjTab T;
    T.ns = tab->ns;
    T.nf = tab->nf;
    T.P = tab->P;
    T.rho_f = tab->rho_f;
    T.F_f = tab->F_f;
    T.phi_f = tab->phi_f;
    T.rc = tab->r_cut;
    AdjIn G;
    G.gE = g_energy;
    G.gF = g_forces;
    G.gW = g_virial;
    double *partialF = ws_at<double>(workspace, L.partialF);
    double *partialP = ws_at<double>(workspace, L.partialP);
    double2 *cc = ws_at<double2>(workspace, L.cc);
    int *cnt = ws_at<int>(workspace, L.cnt);
    int *pos = ws_at<int>(workspace, L.pos);
    int *pairs = ws_at<int>(workspace, L.pairs);
    const int N = sys->n_atoms;
    PROF_BEGIN("eam_adjoint_embed", st);
    eam_adjoint_embed<<<L.gA, EADJ_TA, sizeof(double) * 12 * T.ns, st>>>(S, nl->row_off, nl->upper, nl->nbr, T, G,
                                                                          cc, cnt, partialF);
    MBF_CHECK_LAUNCH();
    int rc = exclusive_scan(cnt, pos, 2 * N, ws_at<int>(workspace, L.scan), st);
    if (rc != MBF_OK) return rc;
    eam_adjoint_compact<<<(N + 127) / 128, 128, 0, st>>>(S, nl->row_off, nl->upper, nl->nbr, T, G, pos, pairs);
    PROF_END("eam_adjoint_embed", st);
    MBF_CHECK_LAUNCH();
    // like pairs [pos[0], pos[N]), cross pairs [pos[N], pos[2 N])
    size_t psm = sizeof(double) * T.ns * T.ns * EADJ_PS;
    int gL = persistent_grid(L.gP, EADJ_TP, (const void *)eam_adjoint_pairs<true>, psm);
    int gC = persistent_grid(L.gP, EADJ_TP, (const void *)eam_adjoint_pairs<false>, psm);
    size_t ni = (size_t)T.ns * T.ns * EADJ_PS;
    PROF_BEGIN("eam_adjoint_pairs", st);
    eam_adjoint_pairs<true><<<gL, EADJ_TP, psm, st>>>(S, nl->row_off, nl->nbr, T, G, cc, pairs, pos, pos + N,
                                                       partialP);
    MBF_CHECK_LAUNCH();
    eam_adjoint_pairs<false><<<gC, EADJ_TP, psm, st>>>(S, nl->row_off, nl->nbr, T, G, cc, pairs, pos + N, pos + 2 * N,
                                                        partialP + (size_t)gL * ni);
    PROF_END("eam_adjoint_pairs", st);
    MBF_CHECK_LAUNCH();
    PROF_BEGIN("eam_adjoint_reduce", st);
    eam_adjoint_final<<<(ne * 32 + 127) / 128, 128, 0, st>>>(T, L.gA, partialF, gL + gC, partialP, d_P);
    PROF_END("eam_adjoint_reduce", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

}  // extern "C"
