// Stillinger-Weber: one kernel for the two-body term and the three-body
// angles of each centre (per-slot forces on the neighbours), then the gather
// through the reverse-slot index.
//
// Replaces engine/stillinger_weber.py:900-1451: single species (:927-1159,
// each unordered neighbour pair once with lambda) and multi species
// (:1165-1451, both orders with lambda/2 of their own (i, j, k) record, legs
// from the pair records (i, j, j)).  The two-body term of a pair reads the
// record of the lower-indexed atom (:714-762).
#include "mbf_util.cuh"

namespace mbf {

// Lanes per atom (LPA) is a template parameter chosen by the host (the
// autotuner); lane groups per block keep the staged rows under 48 KB.
template <int MAXN, int LPA> struct SwGeom {
    static constexpr int GPB = 512 / MAXN;
    static constexpr int BLOCK = GPB * LPA;
};

struct SwDev {
    int ns;
    const double *tb;   // (ns*ns, 8): valid eps sigma a A B p q
    const double *leg;  // (ns*ns, 4): sigma a gamma -
    const double *tri;  // (ns^3, 4):  valid eps*lambda/2 costheta0 -
    double rc;
};

// Three-body term h and its gradient w.r.t. r_ij and r_ik
// (engine/stillinger_weber.py:96-154).
template <typename T>
__device__ __forceinline__ T sw_h3(T rijx, T rijy, T rijz, T r_ij, T rikx, T riky, T rikz, T r_ik, T sig_j,
                                   T a_j, T gam_j, T sig_k, T a_k, T gam_k, T c3, T costh0, T gj[3], T gk[3]) {
    T xij = r_ij / sig_j, xik = r_ik / sig_k;
    if (xij >= a_j || xik >= a_k) {
        gj[0] = gj[1] = gj[2] = gk[0] = gk[1] = gk[2] = T(0);
        return T(0);
    }
    T dj = xij - a_j, dk = xik - a_k;
    T e_ij = clamped_exp<T>(gam_j / dj), e_ik = clamped_exp<T>(gam_k / dk);
    T cos_th = (rijx * rikx + rijy * riky + rijz * rikz) / (r_ij * r_ik);
    T dcos = cos_th - costh0;
    T h = c3 * e_ij * e_ik * dcos * dcos;
    T pre = c3 * e_ij * e_ik * dcos;
    T inv_ij = T(1) / r_ij, inv_ik = T(1) / r_ik;
    T ujx = rijx * inv_ij, ujy = rijy * inv_ij, ujz = rijz * inv_ij;
    T ukx = rikx * inv_ik, uky = riky * inv_ik, ukz = rikz * inv_ik;
    T rad_j = pre * dcos * (-gam_j / (sig_j * dj * dj));
    T rad_k = pre * dcos * (-gam_k / (sig_k * dk * dk));
    T ang_j = T(2) * pre * inv_ij, ang_k = T(2) * pre * inv_ik;
    gj[0] = rad_j * ujx + ang_j * (ukx - cos_th * ujx);
    gj[1] = rad_j * ujy + ang_j * (uky - cos_th * ujy);
    gj[2] = rad_j * ujz + ang_j * (ukz - cos_th * ujz);
    gk[0] = rad_k * ukx + ang_k * (ujx - cos_th * ukx);
    gk[1] = rad_k * uky + ang_k * (ujy - cos_th * uky);
    gk[2] = rad_k * ukz + ang_k * (ujz - cos_th * ukz);
    return h;
}

template <typename T, int MAXN>
struct SwRow {
    T x[MAXN], y[MAXN], z[MAXN], r[MAXN];
    int sp[MAXN];
    int ok[MAXN];
};

// SYM: every (i, j, k) record equals its (i, k, j) twin (one species), so a
// slot needs one h evaluation per partner with the full lambda.
template <typename T, int MAXN, bool SYM, int LPA>
__global__ void sw_force(SysView S, const int *__restrict__ row_off, const int *__restrict__ nbr,
                         const int *__restrict__ rev, SwDev P, double *__restrict__ slot_G, double *__restrict__ f_local,
                         double *__restrict__ per_atom, int *__restrict__ err) {
    constexpr int GPB = SwGeom<MAXN, LPA>::GPB;
    __shared__ SwRow<T, MAXN> rows[GPB];
    const int sub = threadIdx.x & (LPA - 1);
    SwRow<T, MAXN> &R = rows[threadIdx.x / LPA];
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
        if (live) {
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
                R.ok[s] = (r < P.rc && r > 1e-12) ? 1 : 0;
            }
        }
        __syncwarp();
        double fx = 0, fy = 0, fz = 0, e = 0, npair = 0;
        double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (live) {
            int si = S.types[i];
            for (int s = sub; s < n; s += LPA) {
                double Gx = 0, Gy = 0, Gz = 0, cx = 0;
                double dx = (double)R.x[s], dy = (double)R.y[s], dz = (double)R.z[s];
                if (R.ok[s]) {
                    int j = nbr[beg + s];
                    int sj = R.sp[s];
                    int lo = i < j ? si : sj, hi = i < j ? sj : si;
                    // two-body (engine/stillinger_weber.py:23-52)
                    const double *t2 = P.tb + 8 * (lo * ns + hi);
                    T r = R.r[s];
                    if (t2[0] != 0.0) {
                        T sig = (T)t2[2], a = (T)t2[3];
                        T xi_ = r / sig;
                        if (xi_ < a) {
                            T eps = (T)t2[1], A = (T)t2[4], B = (T)t2[5], pp = (T)t2[6], qq = (T)t2[7];
                            T t = T(1) / (xi_ - a);
                            T ex = clamped_exp<T>(t);
                            T xp = RT<T>::pw(xi_, -pp), xq = RT<T>::pw(xi_, -qq);
                            T V2 = eps * A * (B * xp - xq) * ex;
                            T dV2 = eps * A * ex * ((-pp * B * xp / xi_ + qq * xq / xi_) + (B * xp - xq) * (-t * t));
                            e += 0.5 * (double)V2;
                            cx = (double)(dV2 / sig / r);
                        }
                    }
                    // three-body, slot s as one leg of every angle at i
                    const double *ls = P.leg + 4 * (si * ns + sj);
                    T sig_s = (T)ls[0], a_s = (T)ls[1], g_s = (T)ls[2];
                    T gj[3], gk[3];
                    double e3 = 0.0;
                    for (int k = 0; k < n; ++k) {
                        if (k == s || !R.ok[k]) continue;
                        int sk = R.sp[k];
                        const double *lk = P.leg + 4 * (si * ns + sk);
                        const double *t3 = P.tri + 4 * ((si * ns + sj) * ns + sk);
                        if (SYM) {
                            if (t3[0] == 0.0) continue;
                            T h = sw_h3<T>(R.x[s], R.y[s], R.z[s], r, R.x[k], R.y[k], R.z[k], R.r[k], sig_s, a_s,
                                           g_s, (T)lk[0], (T)lk[1], (T)lk[2], T(2) * (T)t3[1], (T)t3[2], gj, gk);
                            e3 += 0.5 * (double)h;
                            Gx -= (double)gj[0];
                            Gy -= (double)gj[1];
                            Gz -= (double)gj[2];
                        } else {
                            if (t3[0] != 0.0) {
                                T h = sw_h3<T>(R.x[s], R.y[s], R.z[s], r, R.x[k], R.y[k], R.z[k], R.r[k], sig_s,
                                               a_s, g_s, (T)lk[0], (T)lk[1], (T)lk[2], (T)t3[1], (T)t3[2], gj, gk);
                                e3 += (double)h;
                                Gx -= (double)gj[0];
                                Gy -= (double)gj[1];
                                Gz -= (double)gj[2];
                            }
                            const double *t3r = P.tri + 4 * ((si * ns + sk) * ns + sj);
                            if (t3r[0] != 0.0) {
                                sw_h3<T>(R.x[k], R.y[k], R.z[k], R.r[k], R.x[s], R.y[s], R.z[s], r, (T)lk[0],
                                         (T)lk[1], (T)lk[2], sig_s, a_s, g_s, (T)t3r[1], (T)t3r[2], gj, gk);
                                Gx -= (double)gk[0];
                                Gy -= (double)gk[1];
                                Gz -= (double)gk[2];
                            }
                        }
                    }
                    e += e3;
                }
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
#pragma unroll
        for (int q = 0; q < 9; ++q) v[q] = group_sum<LPA>(v[q]);
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

template <typename T, int MAXN, bool SYM, int LPA>
static int sw_launch(const SysView &S, const mbf_nlist *nl, const SwDev &P, double *slot_G, double *f_local,
                     double *per_atom, double *forces, int *err, cudaStream_t st) {
    constexpr int GPB = SwGeom<MAXN, LPA>::GPB, BLOCK = SwGeom<MAXN, LPA>::BLOCK;
    int blocks = (S.n_atoms + GPB - 1) / GPB;
    int g = persistent_grid(blocks, BLOCK, (const void *)sw_force<T, MAXN, SYM, LPA>);
    PROF_BEGIN("sw_force", st);
    sw_force<T, MAXN, SYM, LPA><<<g, BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, nl->rev, P, slot_G, f_local, per_atom, err);
    PROF_END("sw_force", st);
    MBF_CHECK_LAUNCH();
    return gather_forces(S.n_atoms, nl->row_off, slot_G, f_local, forces, st);
}

template <typename T, int MAXN, bool SYM>
static int sw_lpa(int lpa, const SysView &S, const mbf_nlist *nl, const SwDev &P, double *slot_G, double *f_local,
                  double *per_atom, double *forces, int *err, cudaStream_t st) {
    switch (lpa) {
        case 4: return sw_launch<T, MAXN, SYM, 4>(S, nl, P, slot_G, f_local, per_atom, forces, err, st);
        case 8: return sw_launch<T, MAXN, SYM, 8>(S, nl, P, slot_G, f_local, per_atom, forces, err, st);
        case 16: return sw_launch<T, MAXN, SYM, 16>(S, nl, P, slot_G, f_local, per_atom, forces, err, st);
        default: return MBF_ERR_ARGUMENT;
    }
}

template <typename T, bool SYM>
static int sw_dispatch(int mr, int lpa, const SysView &S, const mbf_nlist *nl, const SwDev &P, double *slot_G,
                       double *f_local, double *per_atom, double *forces, int *err, cudaStream_t st) {
    if (lpa <= 0) lpa = 8;
    if (mr <= 32) return sw_lpa<T, 32, SYM>(lpa, S, nl, P, slot_G, f_local, per_atom, forces, err, st);
    if (mr <= 64) return sw_lpa<T, 64, SYM>(lpa, S, nl, P, slot_G, f_local, per_atom, forces, err, st);
    return sw_lpa<T, 128, SYM>(lpa, S, nl, P, slot_G, f_local, per_atom, forces, err, st);
}

}  // namespace mbf

using namespace mbf;

extern "C" int mbf_sw_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_sw_tables *tab,
                           const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                           size_t workspace_bytes,
                           double *forces, double *energy, double *virial, void *stream) {
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
    SwDev P;
    P.ns = tab->ns;
    P.tb = tab->tb;
    P.leg = tab->leg;
    P.tri = tab->tri;
    P.rc = tab->r_cut;
    int *err = ws_at<int>(workspace, L.err);
    if (cudaMemsetAsync(err, 0, 16, st) != cudaSuccess) return MBF_ERR_CUDA;
    double *per_atom = ws_at<double>(workspace, L.per_atom);
    double *f_local = ws_at<double>(workspace, L.f_local);
    double *slot_G = ws_at<double>(workspace, L.slot);
    double *partial = ws_at<double>(workspace, L.partial);
    int mr = nl->max_row;
    bool sym = tab->ns == 1;
    int rc;
    if (precision == MBF_FP64)
        rc = sym ? sw_dispatch<double, true>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, st)
                 : sw_dispatch<double, false>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, st);
    else
        rc = sym ? sw_dispatch<float, true>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, st)
                 : sw_dispatch<float, false>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, st);
    if (rc != MBF_OK) return rc;
    return reduce_per_structure(per_atom, plan, sys->n_struct, partial, energy, virial, st);
}
