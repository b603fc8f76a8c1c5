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

constexpr int EADJ_BLOCK = 64;
constexpr int EADJ_NCOL = 43;
constexpr int EADJ_NZ = 20;

struct EamAdjTab {
    int ns, nf;
    const double *P;
    const int *rho_f, *F_f, *phi_f;
    double rc;
};

// pre exp(-expo (x - 1)) / (1 + (x - shift)^20), x = r / re
// (engine/eam_zhou.py:20-45).
template <int K>
__device__ __forceinline__ HD<K> hz_decay(const HD<K> &r, const HD<K> &re, const HD<K> &pre, const HD<K> &expo,
                                          const HD<K> &shift) {
    HD<K> x = r / re;
    HD<K> e = pre * hd_exp<K>((-1.0) * (expo * (x + (-1.0))));
    HD<K> u = x - shift;
    double u2 = u.v * u.v, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8, u18 = u16 * u2;
    HD<K> den = 1.0 + hd_apply<K>(u, u18 * u2, 20.0 * u18 * u.v, 380.0 * u18);
    return e / den;
}

// One element's density f and pair phi_aa (both unswitched) from the 20
// Zhou columns at p; parameter k of the 8 (r_e, f_e, alpha, beta, A, B,
// kappa, lambda) is direction first + k (no direction if out of range).
template <int K>
__device__ __forceinline__ void hz_species(const double *p, int first, const HD<K> &r, HD<K> &f, HD<K> &u) {
    HD<K> re = hd_param<K>(p[0], first + 0, 0), fe = hd_param<K>(p[1], first + 1, 0);
    HD<K> al = hd_param<K>(p[4], first + 2, 0), be = hd_param<K>(p[5], first + 3, 0);
    HD<K> A = hd_param<K>(p[6], first + 4, 0), B = hd_param<K>(p[7], first + 5, 0);
    HD<K> ka = hd_param<K>(p[8], first + 6, 0), la = hd_param<K>(p[9], first + 7, 0);
    HD<K> one = hd_const<K>(1.0);
    HD<K> gB = hz_decay<K>(r, re, one, be, la);
    HD<K> gA = hz_decay<K>(r, re, one, al, ka);
    f = fe * gB;
    u = A * gA - B * gB;
}

// The quintic switch of a row (columns 40, 41) as a function of r only.
template <int K>
__device__ __forceinline__ HD<K> hz_switch(const double *row, const HD<K> &r) {
    double rc = row[2 * EADJ_NZ], w = row[2 * EADJ_NZ + 1];
    double s = (r.v - (rc - w)) / w;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
    double S = 1.0 - s * s * s * (10.0 - 15.0 * s + 6.0 * s * s);
    double dS = -30.0 * s * s * (1.0 - s) * (1.0 - s) / w;
    return hd_apply<K>(r, S, dS, 0.0);  // r carries no parameter direction
}

template <int K, int J>
__device__ __forceinline__ HD<K> hd_lift(const HD<J> &a) {
    HD<K> r = hd_const<K>(a.v);
    r.t = a.t;
    return r;
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

// Site values of atom i into out[0..W).  Returns s_i.
__device__ int eam_atom_sites(const SysView &S, const int *__restrict__ row_off, const int *__restrict__ nbr,
                              const EamAdjTab &T, const AdjIn &G, int i, int W, double *out) {
    const int ns = T.ns;
    for (int w = 0; w < W; ++w) out[w] = 0.0;
    int si = S.types[i];
    int sst = S.n_struct > 1 ? S.atom_struct[i] : 0;
    double gE = G.gE ? G.gE[sst] : 0.0;
    const double *cell = cell_of(S, i);
    const double rc2 = T.rc * T.rc;
    int b = row_off[i], e = row_off[i + 1];
    // pass 1: rho-bar and its tangent
    double rho = 0.0, rho_t = 0.0;
    for (int s = b; s < e; ++s) {
        int j = nbr[s];
        double d[3], r, tg[3];
        adj_leg(S, G, cell, i, j, sst, d, r, tg);
        if (!(r * r < rc2 && r * r > 1e-24)) continue;
        HD<1> rr = hd_const<1>(r);
        rr.t = (d[0] * tg[0] + d[1] * tg[1] + d[2] * tg[2]) / r;
        const double *row = row_of(T, T.rho_f[S.types[j]]);
        HD<1> fs = hz_decay<1>(rr, hd_const<1>(row[0]), hd_const<1>(row[1]), hd_const<1>(row[5]),
                               hd_const<1>(row[9])) *
                   hz_switch<1>(row, rr);
        rho += fs.v;
        rho_t += fs.t;
    }
    // the embedding, rho-bar clamped at 0 as the evaluation does
    double rb = rho > 0.0 ? rho : 0.0;
    HD<13> F = hz_embed(row_of(T, T.F_f[si]), rb, rho_t);
#pragma unroll
    for (int k = 0; k < 12; ++k) out[k] = gE * F.p[k] + F.q[k];
    double c1 = rho > 0.0 ? gE * F.p[12] + F.q[12] : 0.0;
    double c2 = F.p[12];
    // pass 2: density and pair sites per neighbour
    double *dens = out + 12, *pair = out + 12 + 4 * ns;
    for (int s = b; s < e; ++s) {
        int j = nbr[s];
        double d[3], r, tg[3];
        adj_leg(S, G, cell, i, j, sst, d, r, tg);
        if (!(r * r < rc2 && r * r > 1e-24)) continue;
        int sj = S.types[j];
        double rt = (d[0] * tg[0] + d[1] * tg[1] + d[2] * tg[2]) / r;
        {
            HD<4> r4 = hd_const<4>(r);
            r4.t = rt;
            const double *row = row_of(T, T.rho_f[sj]);
            HD<4> re = hd_param<4>(row[0], 0, 0), fe = hd_param<4>(row[1], 1, 0);
            HD<4> be = hd_param<4>(row[5], 2, 0), la = hd_param<4>(row[9], 3, 0);
            HD<4> f = hz_decay<4>(r4, re, fe, be, la) * hz_switch<4>(row, r4);
            double *o = dens + 4 * sj;
#pragma unroll
            for (int k = 0; k < 4; ++k) o[k] += c1 * f.p[k] + c2 * f.q[k];
        }
        HD<8> r8 = hd_const<8>(r);
        r8.t = rt;
        const double *row = row_of(T, T.phi_f[si * ns + sj]);
        HD<8> Sw = hz_switch<8>(row, r8);
        double *o = pair + 17 * sj;
        if (si == sj) {
            HD<8> f, u;
            hz_species<8>(row, 0, r8, f, u);
            HD<8> phi = u * Sw;
#pragma unroll
            for (int k = 0; k < 8; ++k) o[k] += 0.5 * (gE * phi.p[k] + phi.q[k]);
        } else {
            // psi = 1/2 S (q u_a + u_b / q), q = f_b / f_a, phi = k psi
            double kf = row[2 * EADJ_NZ + 2];
            HD<1> r1 = hd_const<1>(r);
            r1.t = rt;
            HD<1> f1, u1;
            HD<8> fa, ua, fb, ub;
            // the earlier species' directions
            hz_species<8>(row, 0, r8, fa, ua);
            hz_species<1>(row + EADJ_NZ, -100, r1, f1, u1);
            fb = hd_lift<8, 1>(f1);
            ub = hd_lift<8, 1>(u1);
            HD<8> q = fb / fa;
            HD<8> psi = 0.5 * (Sw * (q * ua + ub / q));
#pragma unroll
            for (int k = 0; k < 8; ++k) o[k] += 0.5 * kf * (gE * psi.p[k] + psi.q[k]);
            o[16] += 0.5 * (gE * psi.v + psi.t);
            // the later species' directions
            hz_species<1>(row, -100, r1, f1, u1);
            fa = hd_lift<8, 1>(f1);
            ua = hd_lift<8, 1>(u1);
            hz_species<8>(row + EADJ_NZ, 0, r8, fb, ub);
            q = fb / fa;
            psi = 0.5 * (Sw * (q * ua + ub / q));
#pragma unroll
            for (int k = 0; k < 8; ++k) o[8 + k] += 0.5 * kf * (gE * psi.p[k] + psi.q[k]);
        }
    }
    return si;
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

// Sum of entry e = row * 43 + col over `cnt` staged atoms, in atom order.
__device__ double eam_entry_sum(const EamAdjTab &T, int e, int W, int cnt, const double *__restrict__ sm,
                                const int *__restrict__ scode) {
    const int ns = T.ns;
    int f = e / EADJ_NCOL, c = e % EADJ_NCOL;
    double a = 0.0;
    for (int s = 0; s < ns; ++s) {
        if (T.F_f[s] == f) {
            int k = f_site(c);
            if (k >= 0)
                for (int q = 0; q < cnt; ++q)
                    if (scode[q] == s) a += sm[(size_t)q * W + k];
        }
        if (T.rho_f[s] == f) {
            int k = d_site(c);
            if (k >= 0)
                for (int q = 0; q < cnt; ++q)
                    if (scode[q] >= 0) a += sm[(size_t)q * W + 12 + 4 * s + k];
        }
    }
    for (int x = 0; x < ns; ++x)
        for (int y = x; y < ns; ++y) {
            if (T.phi_f[x * ns + y] != f) continue;
            int k = p_site(c);
            if (k < 0 || (x == y && k >= 8)) continue;
            for (int q = 0; q < cnt; ++q) {
                int si = scode[q];
                if (si == x) a += sm[(size_t)q * W + 12 + 4 * ns + 17 * y + k];
                else if (si == y) a += sm[(size_t)q * W + 12 + 4 * ns + 17 * x + k];
            }
        }
    return a;
}

// Block b takes atoms b*EADJ_BLOCK ..: a thread per atom, site values staged
// in shared memory, then the block's sum of every entry to partial[b].
__global__ void __launch_bounds__(EADJ_BLOCK) eam_adjoint_atoms(SysView S, const int *__restrict__ row_off,
                                                                const int *__restrict__ nbr, EamAdjTab T,
                                                                AdjIn G, int W, double *__restrict__ partial) {
    extern __shared__ double sm[];  // EADJ_BLOCK * W site values, then EADJ_BLOCK codes
    int *scode = reinterpret_cast<int *>(sm + (size_t)EADJ_BLOCK * W);
    int i0 = blockIdx.x * EADJ_BLOCK;
    int i = i0 + threadIdx.x;
    int c = -1;
    if (i < S.n_atoms) c = eam_atom_sites(S, row_off, nbr, T, G, i, W, sm + (size_t)threadIdx.x * W);
    scode[threadIdx.x] = c;
    __syncthreads();
    int cnt = min(EADJ_BLOCK, S.n_atoms - i0);
    int ne = T.nf * EADJ_NCOL;
    for (int e = threadIdx.x; e < ne; e += blockDim.x)
        partial[(size_t)blockIdx.x * ne + e] = eam_entry_sum(T, e, W, cnt, sm, scode);
}

// One warp per entry: lanes take every 32nd block partial, then a fixed
// shuffle tree.
__global__ void eam_adjoint_final(int n_blocks, int ne, const double *__restrict__ partial,
                                  double *__restrict__ d_P) {
    int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
    if (e >= ne) return;  // whole warps leave together
    double acc = 0.0;
    for (int b = l; b < n_blocks; b += 32) acc += partial[(size_t)b * ne + e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MBF_FULL, acc, o);
    if (l == 0) d_P[e] = acc;
}

static int eadj_blocks(int n_atoms) { return n_atoms > 0 ? (n_atoms + EADJ_BLOCK - 1) / EADJ_BLOCK : 1; }

}  // namespace mbf

using namespace mbf;

extern "C" {

size_t mbf_eam_adjoint_workspace_bytes(int n_atoms, int nf) {
    if (n_atoms < 0 || nf <= 0) return 0;
    return align256(sizeof(double) * (size_t)eadj_blocks(n_atoms) * nf * EADJ_NCOL);
}

int mbf_eam_adjoint(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab, const double *g_energy,
                    const double *g_forces, const double *g_virial, void *workspace, size_t workspace_bytes,
                    double *d_P, void *stream) {
    if (!sys || !nl || !tab || !workspace || !d_P || tab->ns <= 0 || tab->ns > 8 || tab->nf <= 0)
        return MBF_ERR_ARGUMENT;
    if (nl->n_atoms != sys->n_atoms) return MBF_ERR_ARGUMENT;
    if (workspace_bytes < mbf_eam_adjoint_workspace_bytes(sys->n_atoms, tab->nf)) return MBF_ERR_WORKSPACE;
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
    int W = 12 + 21 * tab->ns;
    size_t smem = (size_t)EADJ_BLOCK * W * sizeof(double) + EADJ_BLOCK * sizeof(int);  // <= 93 KB (ns <= 8)
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(eam_adjoint_atoms, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return MBF_ERR_CUDA;
    int nb = eadj_blocks(sys->n_atoms);
    double *partial = ws_at<double>(workspace, 0);
    PROF_BEGIN("eam_adjoint_atoms", st);
    eam_adjoint_atoms<<<nb, EADJ_BLOCK, smem, st>>>(S, nl->row_off, nl->nbr, T, G, W, partial);
    PROF_END("eam_adjoint_atoms", st);
    MBF_CHECK_LAUNCH();
    PROF_BEGIN("eam_adjoint_reduce", st);
    eam_adjoint_final<<<(ne * 32 + 127) / 128, 128, 0, st>>>(nb, ne, partial, d_P);
    PROF_END("eam_adjoint_reduce", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

}  // extern "C"
