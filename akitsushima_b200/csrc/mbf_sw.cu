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

// Per-leg factors of the three-body term (engine/stillinger_weber.py:96-154):
// h(i, j, k) = c3 E_j E_k (cos theta_jik - cos0)^2 with E_x = exp(gamma_x /
// (r_ix / sigma_x - a_x)) and dE_x/dr_ix = E_x D_x, D_x = -gamma_x /
// (sigma_x (r_ix / sigma_x - a_x)^2).  A leg at or beyond a_x sigma_x has
// E = D = 0, which zeroes every angle it takes part in (the reference's
// early return).  The legs depend only on (centre, neighbour), so they are
// evaluated once per slot, not once per angle.
template <typename T>
__device__ __forceinline__ void sw_leg(T r, T sig, T a, T gam, T &E, T &D) {
    T x = r / sig;
    if (!(x < a)) {
        E = T(0);
        D = T(0);
        return;
    }
    T d = x - a;
    E = clamped_exp<T>(gam / d);
    D = -gam / (sig * d * d);
}

// One centre's row staged in shared memory: displacements, 1/r, leg
// factors, species, and the slots inside the cutoff compacted into `list`.
template <typename T, int MAXN>
struct SwRow {
    T x[MAXN], y[MAXN], z[MAXN], r[MAXN], ir[MAXN], E[MAXN], D[MAXN];
    int sp[MAXN];
    int list[MAXN];
};

// SYM: every (i, j, k) record equals its (i, k, j) twin (one species): one
// coefficient and cos0 for every angle.  Otherwise both orders, each with
// its own record (lambda/2 of (i, j, k) and of (i, k, j)).
//
// For slot s and partner k (both inside the cutoff, k != s) with
// P = E_s E_k, cos = u_s . u_k, dc_o = cos - cos0_o over the orders o:
//   energy booked on slot s:  c_1 P dc_1^2        (order (i, s, k))
//   dh/dr_s = P [D_s A u_s + (B / r_s)(u_k - cos u_s)],
//   A = sum_o c_o dc_o^2,  B = 2 sum_o c_o dc_o,
// so each ordered triple's energy is booked once and each slot collects the
// whole gradient of every angle on its own leg.
template <typename T, int MAXN, bool SYM, int LPA>
__global__ void sw_force(SysView S, const int *__restrict__ row_off, const int *__restrict__ nbr,
                         const int *__restrict__ rev, SwDev P, double *__restrict__ slot_G, double *__restrict__ f_local,
                         double *__restrict__ per_atom, int *__restrict__ err, SiteOut so) {
    constexpr int GPB = SwGeom<MAXN, LPA>::GPB;
    __shared__ SwRow<T, MAXN> rows[GPB];
    const int sub = threadIdx.x & (LPA - 1);
    const int lane = threadIdx.x & 31;
    const unsigned gmask = (LPA == 32) ? 0xffffffffu : (((1u << LPA) - 1u) << (lane & ~(LPA - 1)));
    SwRow<T, MAXN> &R = rows[threadIdx.x / LPA];
    const int ns = P.ns;
    for (int base = blockIdx.x * GPB; base < S.n_atoms; base += gridDim.x * GPB) {
        int i = base + threadIdx.x / LPA;
        int beg = 0, n = 0, nok = 0, si = 0;
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
            si = S.types[i];
            const double *cell = cell_of(S, i);
            double xi = S.pos[3 * (size_t)i], yi = S.pos[3 * (size_t)i + 1], zi = S.pos[3 * (size_t)i + 2];
            // n is uniform over the lane group, so every lane of the group
            // takes the same number of trips and the ballot is complete
            for (int s0 = 0; s0 < n; s0 += LPA) {
                int s = s0 + sub;
                bool ok = false;
                if (s < n) {
                    int j = nbr[beg + s];
                    double dx, dy, dz;
                    mic_exact(cell, S.pos[3 * (size_t)j] - xi, S.pos[3 * (size_t)j + 1] - yi,
                              S.pos[3 * (size_t)j + 2] - zi, dx, dy, dz);
                    double r = sqrt(dx * dx + dy * dy + dz * dz);
                    ok = r < P.rc && r > 1e-12;
                    if (so.vec) {
                        size_t os = 3 * (size_t)(beg + s);
                        so.vec[os] = dx;
                        so.vec[os + 1] = dy;
                        so.vec[os + 2] = dz;
                    }
                    if (ok) {
                        int sj = S.types[j];
                        const double *ls = P.leg + 4 * (si * ns + sj);
                        T E, D;
                        sw_leg<T>((T)r, (T)ls[0], (T)ls[1], (T)ls[2], E, D);
                        R.x[s] = (T)dx;
                        R.y[s] = (T)dy;
                        R.z[s] = (T)dz;
                        R.r[s] = (T)r;
                        R.ir[s] = T(1) / (T)r;
                        R.E[s] = E;
                        R.D[s] = D;
                        R.sp[s] = sj;
                    } else {
                        size_t o = 3 * (size_t)rev[beg + s];
                        slot_G[o] = 0.0;
                        slot_G[o + 1] = 0.0;
                        slot_G[o + 2] = 0.0;
                    }
                }
                unsigned b = __ballot_sync(gmask, ok) >> (lane & ~(LPA - 1));
                if (LPA < 32) b &= (1u << LPA) - 1u;
                if (ok) R.list[nok + __popc(b & ((1u << sub) - 1u))] = s;
                nok += __popc(b);
            }
        }
        __syncwarp();
        double fx = 0, fy = 0, fz = 0, e = 0;
        double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (live) {
            T c_sym = T(0), cos0_sym = T(0);
            if (SYM) {
                c_sym = (T)P.tri[1];
                cos0_sym = (T)P.tri[2];
                if (P.tri[0] == 0.0) c_sym = T(0);
            }
            for (int t = sub; t < nok; t += LPA) {
                int s = R.list[t];
                int j = nbr[beg + s];
                int sj = R.sp[s];
                T xs = R.x[s], ys = R.y[s], zs = R.z[s], r = R.r[s], irs = R.ir[s];
                T Es = R.E[s], Ds = R.D[s];
                double dx = (double)xs, dy = (double)ys, dz = (double)zs;
                double cx = 0.0;
                // two-body (engine/stillinger_weber.py:23-52), record of the
                // lower-indexed atom's species order
                int lo = i < j ? si : sj, hi = i < j ? sj : si;
                const double *t2 = P.tb + 8 * (lo * ns + hi);
                if (t2[0] != 0.0) {
                    T sig = (T)t2[2], a = (T)t2[3];
                    T xi_ = r / sig;
                    if (xi_ < a) {
                        T eps = (T)t2[1], A = (T)t2[4], B = (T)t2[5], pp = (T)t2[6], qq = (T)t2[7];
                        T tt = T(1) / (xi_ - a);
                        T ex = clamped_exp<T>(tt);
                        T xp = RT<T>::pw(xi_, -pp), xq = RT<T>::pw(xi_, -qq);
                        T V2 = eps * A * (B * xp - xq) * ex;
                        T dV2 = eps * A * ex * ((-pp * B * xp / xi_ + qq * xq / xi_) + (B * xp - xq) * (-tt * tt));
                        e += 0.5 * (double)V2;
                        cx = (double)(dV2 / sig / r);
                    }
                }
                // three-body angles with slot s as one leg
                T gx = T(0), gy = T(0), gz = T(0);
                double e3 = 0.0;
                if (Es != T(0)) {
                    for (int u = 0; u < nok; ++u) {
                        if (u == t) continue;
                        int k = R.list[u];
                        T Ek = R.E[k];
                        if (Ek == T(0)) continue;
                        T xk = R.x[k], yk = R.y[k], zk = R.z[k], irk = R.ir[k];
                        T cs = (xs * xk + ys * yk + zs * zk) * (irs * irk);
                        T Pp = Es * Ek;
                        T A, B, eh;
                        if (SYM) {
                            T dc = cs - cos0_sym;
                            eh = c_sym * dc * dc;
                            A = T(2) * eh;
                            B = T(4) * c_sym * dc;
                        } else {
                            int sk = R.sp[k];
                            const double *t3 = P.tri + 4 * ((si * ns + sj) * ns + sk);
                            const double *t3r = P.tri + 4 * ((si * ns + sk) * ns + sj);
                            T c1 = t3[0] != 0.0 ? (T)t3[1] : T(0);
                            T c2 = t3r[0] != 0.0 ? (T)t3r[1] : T(0);
                            T dc1 = cs - (T)t3[2], dc2 = cs - (T)t3r[2];
                            eh = c1 * dc1 * dc1;
                            A = eh + c2 * dc2 * dc2;
                            B = T(2) * (c1 * dc1 + c2 * dc2);
                        }
                        e3 += (double)(Pp * eh);
                        // dh/dr_s = P [(D_s A - B cos / r_s) u_s + (B / r_k) ... ] in
                        // displacement form: u_s = d_s / r_s, u_k = d_k / r_k
                        T as = Pp * (Ds * A - B * cs * irs) * irs;
                        T ak = Pp * B * irs * irk;
                        gx += as * xs + ak * xk;
                        gy += as * ys + ak * yk;
                        gz += as * zs + ak * zk;
                    }
                }
                e += e3;
                double Gx = -(double)gx, Gy = -(double)gy, Gz = -(double)gz;
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
                if (so.dudv) {  // U_i = 1/2 sum V2 + angles at i (engine/site_terms.py:179-300)
                    size_t os = 3 * (size_t)(beg + s);
                    so.dudv[os] = 0.5 * cx * dx - Gx;
                    so.dudv[os + 1] = 0.5 * cx * dy - Gy;
                    so.dudv[os + 2] = 0.5 * cx * dz - Gz;
                }
                // the force on neighbour j goes to j's own slot (j -> i)
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
#pragma unroll
        for (int q = 0; q < 9; ++q) v[q] = group_sum<LPA>(v[q]);
        if (sub == 0 && i < S.n_atoms && so.e) so.e[i] = e;
        if (sub == 0 && i < S.n_atoms) {
            f_local[3 * (size_t)i] = fx;
            f_local[3 * (size_t)i + 1] = fy;
            f_local[3 * (size_t)i + 2] = fz;
            double *pa = per_atom + (size_t)i * ATOM_ACC;
            pa[0] = e;
#pragma unroll
            for (int q = 0; q < 9; ++q) pa[1 + q] = v[q];
            pa[10] = (double)nok;
        }
        __syncwarp();
    }
}

template <typename T, int MAXN, bool SYM, int LPA>
static int sw_launch(const SysView &S, const mbf_nlist *nl, const SwDev &P, double *slot_G, double *f_local,
                     double *per_atom, double *forces, int *err, const SiteOut &so, cudaStream_t st) {
    constexpr int GPB = SwGeom<MAXN, LPA>::GPB, BLOCK = SwGeom<MAXN, LPA>::BLOCK;
    int blocks = (S.n_atoms + GPB - 1) / GPB;
    int g = persistent_grid(blocks, BLOCK, (const void *)sw_force<T, MAXN, SYM, LPA>);
    PROF_BEGIN("sw_force", st);
    sw_force<T, MAXN, SYM, LPA><<<g, BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, nl->rev, P, slot_G, f_local, per_atom, err,
                                                     so);
    PROF_END("sw_force", st);
    MBF_CHECK_LAUNCH();
    return MBF_OK;   // the eval's gather_reduce adds the slot forces
}

template <typename T, int MAXN, bool SYM>
static int sw_lpa(int lpa, const SysView &S, const mbf_nlist *nl, const SwDev &P, double *slot_G, double *f_local,
                  double *per_atom, double *forces, int *err, const SiteOut &so, cudaStream_t st) {
    switch (lpa) {
        case 4: return sw_launch<T, MAXN, SYM, 4>(S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
        case 8: return sw_launch<T, MAXN, SYM, 8>(S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
        case 16: return sw_launch<T, MAXN, SYM, 16>(S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
        default: return MBF_ERR_ARGUMENT;
    }
}

template <typename T, bool SYM>
static int sw_dispatch(int mr, int lpa, const SysView &S, const mbf_nlist *nl, const SwDev &P, double *slot_G,
                       double *f_local, double *per_atom, double *forces, int *err, const SiteOut &so,
                       cudaStream_t st) {
    if (lpa <= 0) lpa = 8;
    if (mr <= 32) return sw_lpa<T, 32, SYM>(lpa, S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
    if (mr <= 64) return sw_lpa<T, 64, SYM>(lpa, S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
    return sw_lpa<T, 128, SYM>(lpa, S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
}

}  // namespace mbf

using namespace mbf;

static int sw_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_sw_tables *tab,
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
    SwDev P;
    P.ns = tab->ns;
    P.tb = tab->tb;
    P.leg = tab->leg;
    P.tri = tab->tri;
    P.rc = tab->r_cut;
    int *err = ws_at<int>(workspace, L.err);
    if (cudaMemsetAsync(err, 0, ERR_CLEAR_BYTES, st) != cudaSuccess) return MBF_ERR_CUDA;
    double *per_atom = ws_at<double>(workspace, L.per_atom);
    double *f_local = ws_at<double>(workspace, L.f_local);
    double *slot_G = ws_at<double>(workspace, L.slot);
    double *partial = ws_at<double>(workspace, L.partial);
    int mr = nl->max_row;
    bool sym = tab->ns == 1;
    int rc;
    if (precision == MBF_FP64)
        rc = sym ? sw_dispatch<double, true>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, so, st)
                 : sw_dispatch<double, false>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
    else
        rc = sym ? sw_dispatch<float, true>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, so, st)
                 : sw_dispatch<float, false>(mr, lanes_per_atom, S, nl, P, slot_G, f_local, per_atom, forces, err, so, st);
    if (rc != MBF_OK) return rc;
    return gather_reduce(sys->n_struct, sys->n_atoms, nl->row_off, slot_G, f_local, forces, per_atom, plan, partial,
                         energy, virial, ws_at<unsigned>(workspace, L.sdone), st);
}

extern "C" int mbf_sw_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_sw_tables *tab,
                           const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                           size_t workspace_bytes, double *forces, double *energy, double *virial, void *stream) {
    SiteOut none = {nullptr, nullptr, nullptr};
    return sw_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, forces, energy, virial,
                   none, stream);
}

extern "C" int mbf_sw_eval_sites(const mbf_system *sys, const mbf_nlist *nl, const mbf_sw_tables *tab,
                                 const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                                 size_t workspace_bytes, double *forces, double *energy, double *virial,
                                 double *site_e, double *site_dudv, double *site_vec, void *stream) {
    if (!site_e || !site_dudv || !site_vec) return MBF_ERR_ARGUMENT;
    if (nl && nl->n_slots > 0 &&
        cudaMemsetAsync(site_dudv, 0, sizeof(double) * 3 * (size_t)nl->n_slots, (cudaStream_t)stream) != cudaSuccess)
        return MBF_ERR_CUDA;
    SiteOut so = {site_e, site_dudv, site_vec};
    return sw_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, forces, energy, virial,
                   so, stream);
}
