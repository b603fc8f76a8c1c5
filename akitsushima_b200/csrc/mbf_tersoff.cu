// Tersoff bond-order potential: zeta/bond-order kernel, force kernel with
// per-slot three-body forces, gather through the reverse-slot index.
//
// Replaces engine/tersoff.py:1208-1711 (single-species :1233-1513 with m = 3
// and gamma = 1, multi-species :1518-1711 with its dense species tables
// :1606-1653).  Energy E = sum_{i<j} fc (fR + b_avg fA), b_avg the mean of
// the two bond orders (engine/tersoff.py:6-19).
//
// Owner computes, no atomics: the lane group of centre i evaluates every
// zeta-term gradient of its angles, keeps the force on i and writes the force
// its angles put on neighbour x into x's own slot (x -> i); atom a later sums
// its own row of slots (gather_reduce).
#include "mbf_util.cuh"

namespace mbf {

// Lanes per atom (LPA) is a template parameter chosen by the host (the
// autotuner); lane groups per block keep the staged rows under 48 KB.
template <int MAXN, int LPA> struct TeGeom {
    static constexpr int GPB = 512 / MAXN;
    static constexpr int BLOCK = GPB * LPA;
};

struct TeDev {
    int ns;
    const double *tb;   // (ns*ns, 10): valid A B l1 l2 R D beta n -
    const double *tri;  // (ns^3, 8):   valid c d h l3 m gam -
    double rc;
};

template <typename T>
__device__ __forceinline__ T te_fc(T r, T R, T D) {
    if (r < R - D) return T(1);
    if (r > R + D) return T(0);
    return T(0.5) - T(0.5) * RT<T>::sn(T(0.5) * T(3.14159265358979323846) * (r - R) / D);
}

template <typename T>
__device__ __forceinline__ T te_dfc(T r, T R, T D) {
    if (r < R - D || r > R + D) return T(0);
    return T(-0.25) * T(3.14159265358979323846) / D * RT<T>::cs(T(0.5) * T(3.14159265358979323846) * (r - R) / D);
}

// (l3 u)^m for m = 1 or 3 by multiplication, pow otherwise.
template <typename T>
__device__ __forceinline__ T te_arg(T l3, T u, T m) {
    if (m == T(3)) return (l3 * l3 * l3) * (u * u * u);
    if (m == T(1)) return l3 * u;
    return RT<T>::pw(l3, m) * RT<T>::pw(u, m);
}

// Angular function g = 1 + c^2/d^2 - c^2/(d^2 + (h - cos)^2), written as
// 1 + c^2 (h - cos)^2 / (d^2 (d^2 + (h - cos)^2)): the same value without
// the cancellation of two ~c^2/d^2 terms (c^2/d^2 ~ 4e7 for silicon), which
// float32 cannot afford.
template <typename T>
__device__ __forceinline__ T te_g(T c, T d, T hc) {
    T d2 = d * d, hc2 = hc * hc;
    return T(1) + (c * c) * hc2 / (d2 * (d2 + hc2));
}

// Analytic gradient of one zeta term (engine/tersoff.py:161-202).
template <typename T>
__device__ __forceinline__ void te_zgrad(T rijx, T rijy, T rijz, T r_ij, T rikx, T riky, T rikz, T r_ik,
                                         T fc_ik, T dfc_ik, T c, T d, T h, T l3, T m, T gam, T dzj[3],
                                         T dzk[3]) {
    T inv_ij = T(1) / r_ij, inv_ik = T(1) / r_ik;
    T cos_t = (rijx * rikx + rijy * riky + rijz * rikz) * inv_ij * inv_ik;
    T hc = h - cos_t;
    T q = d * d + hc * hc;
    T g = te_g<T>(c, d, hc);
    T dg = T(-2) * c * c * hc / (q * q);
    T u = r_ij - r_ik;
    T ex = clamped_exp<T>(te_arg<T>(l3, u, m));
    T dex;
    if (m == T(3)) dex = ex * T(3) * (l3 * l3 * l3) * (u * u);
    else if (m == T(1)) dex = ex * l3;
    else dex = ex * m * RT<T>::pw(l3, m) * RT<T>::pw(u, m - T(1));
    T a_j = gam * fc_ik * dg * ex;
    T b_j = gam * fc_ik * g * dex * inv_ij;
    T b_k = gam * (dfc_ik * g * ex - fc_ik * g * dex) * inv_ik;
    T ii_k = inv_ij * inv_ik;
    T cj = cos_t * inv_ij * inv_ij;
    T ck = cos_t * inv_ik * inv_ik;
    dzj[0] = a_j * (rikx * ii_k - cj * rijx) + b_j * rijx;
    dzj[1] = a_j * (riky * ii_k - cj * rijy) + b_j * rijy;
    dzj[2] = a_j * (rikz * ii_k - cj * rijz) + b_j * rijz;
    dzk[0] = a_j * (rijx * ii_k - ck * rikx) + b_k * rikx;
    dzk[1] = a_j * (rijy * ii_k - ck * riky) + b_k * riky;
    dzk[2] = a_j * (rijz * ii_k - ck * rikz) + b_k * rikz;
}

// Shared-memory row staging of one lane group.
template <typename T, int MAXN>
struct TeRow {
    T x[MAXN], y[MAXN], z[MAXN], r[MAXN], coef[MAXN];
    int sp[MAXN];
    int ok[MAXN];
};

template <typename T, int MAXN, int LPA>
__device__ __forceinline__ void te_stage(const SysView &S, const int *__restrict__ nbr, int i, int beg,
                                         int n, double rc, TeRow<T, MAXN> &R, int sub) {
    const double *cell = cell_of(S, i);
    double xi = S.pos[3 * (size_t)i], yi = S.pos[3 * (size_t)i + 1], zi = S.pos[3 * (size_t)i + 2];
    for (int s = sub; s < n; s += LPA) {
        int j = nbr[beg + s];
        double dx, dy, dz;
        mic_exact(cell, S.pos[3 * (size_t)j] - xi, S.pos[3 * (size_t)j + 1] - yi,
                  S.pos[3 * (size_t)j + 2] - zi, dx, dy, dz);
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        R.x[s] = (T)dx;
        R.y[s] = (T)dy;
        R.z[s] = (T)dz;
        R.r[s] = (T)r;
        R.sp[s] = S.types[j];
        R.ok[s] = (r < rc && r > 1e-12) ? 1 : 0;
    }
}

template <typename T, int MAXN, int LPA>
__global__ void te_zeta(SysView S, const int *__restrict__ row_off, const int *__restrict__ nbr, TeDev P,
                        double *__restrict__ slot_b, int *__restrict__ err) {
    constexpr int GPB = TeGeom<MAXN, LPA>::GPB;
    __shared__ TeRow<T, MAXN> rows[GPB];
    const int sub = threadIdx.x & (LPA - 1);
    TeRow<T, MAXN> &R = rows[threadIdx.x / LPA];
    const int ns = P.ns;
    for (int base = blockIdx.x * GPB; base < S.n_atoms; base += gridDim.x * GPB) {
        int i = base + threadIdx.x / LPA;
        int beg = 0, n = 0;
        bool live = i < S.n_atoms;
        if (live) {
            beg = row_off[i];
            n = row_off[i + 1] - beg;
            if (n > MAXN) {
                if (sub == 0) atomicOr(err, MBF_DEV_ROW_TOO_LONG);
                live = false;
            }
        }
        if (live) te_stage<T, MAXN, LPA>(S, nbr, i, beg, n, P.rc, R, sub);
        __syncwarp();
        if (live) {
            int si = S.types[i];
            for (int s = sub; s < n; s += LPA) {
                double b = 1.0, db = 0.0;
                if (R.ok[s]) {
                    int j = nbr[beg + s];
                    int sj = R.sp[s];
                    int lo = i < j ? si : sj, hi = i < j ? sj : si;
                    if (P.tb[10 * (lo * ns + hi)] != 0.0) {
                        T zeta = T(0);
                        T rs = R.r[s];
                        for (int k = 0; k < n; ++k) {
                            if (k == s || !R.ok[k]) continue;
                            int sk = R.sp[k];
                            const double *tk = P.tb + 10 * (si * ns + sk);
                            const double *t3 = P.tri + 8 * ((si * ns + sj) * ns + sk);
                            if (tk[0] == 0.0 || t3[0] == 0.0) continue;
                            T fc = te_fc<T>(R.r[k], (T)tk[5], (T)tk[6]);
                            if (fc == T(0)) continue;
                            T cos_t = (R.x[s] * R.x[k] + R.y[s] * R.y[k] + R.z[s] * R.z[k]) / (rs * R.r[k]);
                            T c = (T)t3[1], d = (T)t3[2], h = (T)t3[3];
                            T hc = h - cos_t;
                            T g = te_g<T>(c, d, hc);
                            zeta += (T)t3[6] * fc * g * clamped_exp<T>(te_arg<T>((T)t3[4], rs - R.r[k], (T)t3[5]));
                        }
                        const double *tij = P.tb + 10 * (si * ns + sj);
                        double beta = tij[7], nn = tij[8];
                        double z = (double)zeta;
                        if (z > 0.0 && beta != 0.0) {
                            double bz = pow(beta * z, nn);
                            b = pow(1.0 + bz, -0.5 / nn);
                            db = -0.5 * b * bz / (z * (1.0 + bz));
                        }
                    }
                }
                slot_b[2 * (size_t)(beg + s)] = b;
                slot_b[2 * (size_t)(beg + s) + 1] = db;
            }
        }
        __syncwarp();
    }
}

template <typename T, int MAXN, int LPA>
__global__ void te_force(SysView S, const int *__restrict__ row_off, const int *__restrict__ nbr,
                         const int *__restrict__ rev, TeDev P, const double *__restrict__ slot_b,
                         double *__restrict__ slot_G, double *__restrict__ f_local,
                         double *__restrict__ per_atom, int *__restrict__ err, SiteOut so) {
    constexpr int GPB = TeGeom<MAXN, LPA>::GPB;
    __shared__ TeRow<T, MAXN> rows[GPB];
    const int sub = threadIdx.x & (LPA - 1);
    TeRow<T, MAXN> &R = rows[threadIdx.x / LPA];
    const int ns = P.ns;
    for (int base = blockIdx.x * GPB; base < S.n_atoms; base += gridDim.x * GPB) {
        int i = base + threadIdx.x / LPA;
        int beg = 0, n = 0;
        bool live = i < S.n_atoms;
        if (live) {
            beg = row_off[i];
            n = row_off[i + 1] - beg;
            if (n > MAXN) {
                if (sub == 0) atomicOr(err, MBF_DEV_ROW_TOO_LONG);
                live = false;
            }
        }
        if (live) te_stage<T, MAXN, LPA>(S, nbr, i, beg, n, P.rc, R, sub);
        __syncwarp();
        double fx = 0, fy = 0, fz = 0, e = 0, npair = 0, e_site = 0;
        double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        int si = live ? S.types[i] : 0;
        // pass 1: pair terms and the zeta-gradient coefficients
        double cxs[(MAXN + LPA - 1) / LPA];
        double cxs_site[(MAXN + LPA - 1) / LPA];  // site split: own bond order (engine/site_terms.py:312-437)
        double pair_r[(MAXN + LPA - 1) / LPA];
        if (live) {
            const double *cell = cell_of(S, i);
            double xi = S.pos[3 * (size_t)i], yi = S.pos[3 * (size_t)i + 1], zi = S.pos[3 * (size_t)i + 2];
            int q = 0;
            for (int s = sub; s < n; s += LPA, ++q) {
                {
                    int j = nbr[beg + s];
                    double dx, dy, dz;
                    mic_exact(cell, S.pos[3 * (size_t)j] - xi, S.pos[3 * (size_t)j + 1] - yi,
                              S.pos[3 * (size_t)j + 2] - zi, dx, dy, dz);
                    pair_r[q] = sqrt(dx * dx + dy * dy + dz * dz);
                }
                T coef = T(0);
                double cx = 0.0, cx_site = 0.0;
                if (R.ok[s]) {
                    int j = nbr[beg + s];
                    int sj = R.sp[s];
                    int lo = i < j ? si : sj, hi = i < j ? sj : si;
                    const double *tp = P.tb + 10 * (lo * ns + hi);
                    if (tp[0] != 0.0) {
                        double b_own = slot_b[2 * (size_t)(beg + s)];
                        double db_own = slot_b[2 * (size_t)(beg + s) + 1];
                        double b_rev = slot_b[2 * (size_t)rev[beg + s]];
                        double bavg = i < j ? 0.5 * (b_own + b_rev) : 0.5 * (b_rev + b_own);
                        // the two-body part is per bond, not per angle: float64
                        // in both precisions
                        double r = pair_r[q];
                        double Rr = tp[5], Dd = tp[6];
                        double fc = te_fc<double>(r, Rr, Dd), dfc = te_dfc<double>(r, Rr, Dd);
                        if (fc != 0.0 || dfc != 0.0) {
                            double l1 = tp[3], l2 = tp[4];
                            double fr = tp[1] * clamped_exp<double>(-l1 * r);
                            double fa = -tp[2] * clamped_exp<double>(-l2 * r);
                            e += 0.5 * (fc * (fr + bavg * fa));
                            double dEdr = dfc * (fr + bavg * fa) + fc * (-l1 * fr + bavg * (-l2 * fa));
                            cx = dEdr / r;
                            if (so.dudv) {
                                e_site += 0.5 * (fc * (fr + b_own * fa));
                                cx_site = 0.5 * (dfc * (fr + b_own * fa) + fc * (-l1 * fr - l2 * b_own * fa)) / r;
                            }
                            if (fabs(db_own) > 1e-30) coef = (T)(0.5 * fc * fa * db_own);
                        }
                    }
                }
                R.coef[s] = coef;
                cxs[q] = cx;
                cxs_site[q] = cx_site;
            }
        }
        __syncwarp();
        // pass 2: three-body forces per slot
        if (live) {
            int q = 0;
            for (int s = sub; s < n; s += LPA, ++q) {
                double Gx = 0, Gy = 0, Gz = 0;
                double dx = (double)R.x[s], dy = (double)R.y[s], dz = (double)R.z[s];
                if (R.ok[s]) {
                    int sx_ = R.sp[s];
                    T dzj[3], dzk[3];
                    // slot s as the bond partner j of zeta_{i s}
                    T cs = R.coef[s];
                    if (cs != T(0)) {
                        for (int k = 0; k < n; ++k) {
                            if (k == s || !R.ok[k]) continue;
                            int sk = R.sp[k];
                            const double *tk = P.tb + 10 * (si * ns + sk);
                            const double *t3 = P.tri + 8 * ((si * ns + sx_) * ns + sk);
                            if (tk[0] == 0.0 || t3[0] == 0.0) continue;
                            T Rk = (T)tk[5], Dk = (T)tk[6];
                            T fck = te_fc<T>(R.r[k], Rk, Dk);
                            if (fck == T(0)) continue;
                            te_zgrad<T>(R.x[s], R.y[s], R.z[s], R.r[s], R.x[k], R.y[k], R.z[k], R.r[k], fck,
                                        te_dfc<T>(R.r[k], Rk, Dk), (T)t3[1], (T)t3[2], (T)t3[3], (T)t3[4],
                                        (T)t3[5], (T)t3[6], dzj, dzk);
                            Gx -= (double)(cs * dzj[0]);
                            Gy -= (double)(cs * dzj[1]);
                            Gz -= (double)(cs * dzj[2]);
                        }
                    }
                    // slot s as the third atom k of zeta_{i j}
                    const double *ts = P.tb + 10 * (si * ns + sx_);
                    if (ts[0] != 0.0) {
                        T Rs = (T)ts[5], Ds = (T)ts[6];
                        T fcs = te_fc<T>(R.r[s], Rs, Ds);
                        if (fcs != T(0)) {
                            T dfcs = te_dfc<T>(R.r[s], Rs, Ds);
                            for (int jj = 0; jj < n; ++jj) {
                                if (jj == s || !R.ok[jj]) continue;
                                T cj = R.coef[jj];
                                if (cj == T(0)) continue;
                                const double *t3 = P.tri + 8 * ((si * ns + R.sp[jj]) * ns + sx_);
                                if (t3[0] == 0.0) continue;
                                te_zgrad<T>(R.x[jj], R.y[jj], R.z[jj], R.r[jj], R.x[s], R.y[s], R.z[s], R.r[s],
                                            fcs, dfcs, (T)t3[1], (T)t3[2], (T)t3[3], (T)t3[4], (T)t3[5],
                                            (T)t3[6], dzj, dzk);
                                Gx -= (double)(cj * dzk[0]);
                                Gy -= (double)(cj * dzk[1]);
                                Gz -= (double)(cj * dzk[2]);
                            }
                        }
                    }
                }
                double cx = cxs[q];
                fx += cx * dx - Gx;
                fy += cx * dy - Gy;
                fz += cx * dz - Gz;
                double hx = 0.5 * cx * dx, hy = 0.5 * cx * dy, hz = 0.5 * cx * dz;
                v[0] += -hx * dx + Gx * dx;
                v[1] += -hx * dy + Gx * dy;
                v[2] += -hx * dz + Gx * dz;
                v[3] += -hy * dx + Gy * dx;
                v[4] += -hy * dy + Gy * dy;
                v[5] += -hy * dz + Gy * dz;
                v[6] += -hz * dx + Gz * dx;
                v[7] += -hz * dy + Gz * dy;
                v[8] += -hz * dz + Gz * dz;
                npair += R.ok[s] ? 1.0 : 0.0;
                if (so.dudv) {
                    size_t os = 3 * (size_t)(beg + s);
                    double cs_ = cxs_site[q];
                    so.dudv[os] = cs_ * dx - Gx;
                    so.dudv[os + 1] = cs_ * dy - Gy;
                    so.dudv[os + 2] = cs_ * dz - Gz;
                    so.vec[os] = dx;
                    so.vec[os + 1] = dy;
                    so.vec[os + 2] = dz;
                }
                // the force on neighbour x goes to x's own slot (x -> i)
                size_t o = 3 * (size_t)rev[beg + s];
                slot_G[o] = Gx;
                slot_G[o + 1] = Gy;
                slot_G[o + 2] = Gz;
            }
        }
        fx = group_sum<LPA>(fx);
        fy = group_sum<LPA>(fy);
        fz = group_sum<LPA>(fz);
        e = group_sum<LPA>(e);
        npair = group_sum<LPA>(npair);
        e_site = group_sum<LPA>(e_site);
#pragma unroll
        for (int q = 0; q < 9; ++q) v[q] = group_sum<LPA>(v[q]);
        if (sub == 0 && i < S.n_atoms && so.e) so.e[i] = e_site;
        if (sub == 0 && i < S.n_atoms) {
            f_local[3 * (size_t)i] = fx;
            f_local[3 * (size_t)i + 1] = fy;
            f_local[3 * (size_t)i + 2] = fz;
            double *pa = per_atom + (size_t)i * ATOM_ACC;
            pa[0] = e;
#pragma unroll
            for (int q = 0; q < 9; ++q) pa[1 + q] = v[q];
            pa[10] = npair;
        }
        __syncwarp();
    }
}

template <typename T, int MAXN, int LPA>
static int te_launch(const SysView &S, const mbf_nlist *nl, const TeDev &P, double *slot_b, double *slot_G,
                     double *f_local, double *per_atom, double *forces, int *err, const SiteOut &so,
                     cudaStream_t st) {
    constexpr int GPB = TeGeom<MAXN, LPA>::GPB, BLOCK = TeGeom<MAXN, LPA>::BLOCK;
    int blocks = (S.n_atoms + GPB - 1) / GPB;
    int g = persistent_grid(blocks, BLOCK, (const void *)te_zeta<T, MAXN, LPA>);
    PROF_BEGIN("te_zeta", st);
    te_zeta<T, MAXN, LPA><<<g, BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, P, slot_b, err);
    PROF_END("te_zeta", st);
    MBF_CHECK_LAUNCH();
    g = persistent_grid(blocks, BLOCK, (const void *)te_force<T, MAXN, LPA>);
    PROF_BEGIN("te_force", st);
    te_force<T, MAXN, LPA><<<g, BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, nl->rev, P, slot_b, slot_G, f_local,
                                         per_atom, err, so);
    PROF_END("te_force", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;   // the eval's gather_reduce adds the slot forces
}

template <typename T, int MAXN>
static int te_lpa(int lpa, const SysView &S, const mbf_nlist *nl, const TeDev &P, double *slot_b,
                  double *slot_G, double *f_local, double *per_atom, double *forces, int *err, const SiteOut &so,
                  cudaStream_t st) {
    switch (lpa) {
        case 4: return te_launch<T, MAXN, 4>(S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st);
        case 8: return te_launch<T, MAXN, 8>(S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st);
        case 16: return te_launch<T, MAXN, 16>(S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st);
        default: return MBF_ERR_ARGUMENT;
    }
}

template <typename T>
static int te_rows(int mr, int lpa, const SysView &S, const mbf_nlist *nl, const TeDev &P, double *slot_b,
                   double *slot_G, double *f_local, double *per_atom, double *forces, int *err, const SiteOut &so,
                   cudaStream_t st) {
    if (mr <= 32) return te_lpa<T, 32>(lpa, S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st);
    if (mr <= 64) return te_lpa<T, 64>(lpa, S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st);
    return te_lpa<T, 128>(lpa, S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st);
}

static int te_dispatch(int precision, int mr, int lpa, const SysView &S, const mbf_nlist *nl, const TeDev &P,
                       double *slot_b, double *slot_G, double *f_local, double *per_atom, double *forces,
                       int *err, const SiteOut &so, cudaStream_t st) {
    if (lpa <= 0) lpa = 8;
    return precision == MBF_FP64
               ? te_rows<double>(mr, lpa, S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st)
               : te_rows<float>(mr, lpa, S, nl, P, slot_b, slot_G, f_local, per_atom, forces, err, so, st);
}

}  // namespace mbf

using namespace mbf;

static int tersoff_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_tersoff_tables *tab,
                        const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                        size_t workspace_bytes, double *forces, double *energy, double *virial, const SiteOut &so,
                        void *stream) {
    if (!sys || !nl || !tab || !plan || !workspace || !forces || !energy || !virial) return MBF_ERR_ARGUMENT;
    if (precision != MBF_FP64 && precision != MBF_MIXED) return MBF_ERR_ARGUMENT;
    if (nl->n_atoms != sys->n_atoms || tab->ns <= 0) return MBF_ERR_ARGUMENT;
    EvalLayout L = eval_layout(sys->n_atoms, nl->n_slots, plan->n_chunks);
    if (workspace_bytes < L.total) return MBF_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    if (sys->n_atoms == 0) {
        if (cudaMemsetAsync(energy, 0, sizeof(double) * sys->n_struct, st) != cudaSuccess) return MBF_ERR_CUDA;
        if (cudaMemsetAsync(virial, 0, sizeof(double) * 9 * sys->n_struct, st) != cudaSuccess) return MBF_ERR_CUDA;
        return MBF_OK;
    }
    if (nl->max_row > 128) return MBF_ERR_ROW_TOO_LONG;
    SysView S = make_view(sys);
    TeDev P;
    P.ns = tab->ns;
    P.tb = tab->tb;
    P.tri = tab->tri;
    P.rc = tab->r_cut;
    int *err = ws_at<int>(workspace, L.err);
    if (cudaMemsetAsync(err, 0, ERR_CLEAR_BYTES, st) != cudaSuccess) return MBF_ERR_CUDA;
    double *per_atom = ws_at<double>(workspace, L.per_atom);
    double *f_local = ws_at<double>(workspace, L.f_local);
    double *slot_G = ws_at<double>(workspace, L.slot);
    double *slot_b = ws_at<double>(workspace, L.slot_b);
    double *partial = ws_at<double>(workspace, L.partial);
    int rc = te_dispatch(precision, nl->max_row, lanes_per_atom, S, nl, P, slot_b, slot_G, f_local, per_atom,
                         forces, err, so, st);
    if (rc != MBF_OK) return rc;
    return gather_reduce(sys->n_struct, sys->n_atoms, nl->row_off, slot_G, f_local, forces, per_atom, plan, partial,
                         energy, virial, ws_at<unsigned>(workspace, L.sdone), st);
}

extern "C" int mbf_tersoff_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_tersoff_tables *tab,
                                const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                                size_t workspace_bytes, double *forces, double *energy, double *virial,
                                void *stream) {
    SiteOut none = {nullptr, nullptr, nullptr};
    return tersoff_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, forces, energy,
                        virial, none, stream);
}

extern "C" int mbf_tersoff_eval_sites(const mbf_system *sys, const mbf_nlist *nl, const mbf_tersoff_tables *tab,
                                      const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                                      void *workspace, size_t workspace_bytes, double *forces, double *energy,
                                      double *virial, double *site_e, double *site_dudv, double *site_vec,
                                      void *stream) {
    if (!site_e || !site_dudv || !site_vec) return MBF_ERR_ARGUMENT;
    if (nl && nl->n_slots > 0 &&
        cudaMemsetAsync(site_dudv, 0, sizeof(double) * 3 * (size_t)nl->n_slots, (cudaStream_t)stream) != cudaSuccess)
        return MBF_ERR_CUDA;
    SiteOut so = {site_e, site_dudv, site_vec};
    return tersoff_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, forces, energy,
                        virial, so, stream);
}
