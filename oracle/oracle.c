/*
 * CPU oracle for the many-body force path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the numba kernels of the reference
 * (akitsushima 0.4.0a4) that the CUDA path replaces.  Each function cites the
 * reference file:line it follows and keeps that function's loop order and
 * arithmetic, so its results agree with the reference to rounding (the
 * reference's numba kernels are compiled with fastmath, this file is not).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * the shared library built from this file.  The product (akitsushima_b200)
 * never links or calls it.
 *
 * Threading: the loops the reference runs under numba prange run here under
 * OpenMP with per-thread force buffers (the reference's own pattern,
 * engine/tersoff.py:328-461).  With one thread every function is serial.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared).
 * -ffp-contract=off keeps a*b+c as two rounded operations, which is what the
 * neighbour-list pair test needs to reproduce the reference bit for bit
 * (engine/neighborlist.py:376-380: that kernel is compiled without fastmath).
 */
#include <math.h>
#define ORC_PI 3.14159265358979323846
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static int orc_tid(void) {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

int orc_num_threads(void) { return orc_threads(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* engine/_numba_common.py:12-33 -- exp clamped at +-500. */
static double nb_exp(double x) {
    static double hi = 0.0;
    if (hi == 0.0) hi = exp(500.0);
    if (x > 500.0) return hi;
    if (x < -500.0) return 0.0;
    return exp(x);
}

/* ------------------------------------------------------------------ */
/* Neighbour list                                                       */
/* ------------------------------------------------------------------ */

/* engine/neighborlist.py:312-373 (_cell_linked_pairs_numpy).  Pair (i, j) is
 * kept iff j > i, r2 < rl2 and r2 > 1e-20 after the minimum-image reduction
 * s -= round(s), round = round-half-even (numba lowers round() to llvm.rint).
 * Returns the number of pairs; with count_only the out_* arrays are unused. */
long orc_cll_pairs(long N, long nc0, long nc1, long nc2,
                   const long *cell_idx, const long *offsets, long n_offsets,
                   const long *head, const long *nxt,
                   const double *pos, const double *lat, const double *inv,
                   double rl2, int *out_i, int *out_j, double *out_rij,
                   double *out_r, int count_only)
{
    long n_found = 0;
    for (long i = 0; i < N; ++i) {
        long ci0 = cell_idx[3 * i], ci1 = cell_idx[3 * i + 1], ci2 = cell_idx[3 * i + 2];
        for (long o = 0; o < n_offsets; ++o) {
            long cj0 = (ci0 + offsets[3 * o]) % nc0;
            long cj1 = (ci1 + offsets[3 * o + 1]) % nc1;
            long cj2 = (ci2 + offsets[3 * o + 2]) % nc2;
            if (cj0 < 0) cj0 += nc0;   /* python % is non-negative */
            if (cj1 < 0) cj1 += nc1;
            if (cj2 < 0) cj2 += nc2;
            long cflat = cj0 * nc1 * nc2 + cj1 * nc2 + cj2;
            for (long j = head[cflat]; j >= 0; j = nxt[j]) {
                if (j <= i) continue;
                double rx = pos[3 * j] - pos[3 * i];
                double ry = pos[3 * j + 1] - pos[3 * i + 1];
                double rz = pos[3 * j + 2] - pos[3 * i + 2];
                double sx = rx * inv[0] + ry * inv[3] + rz * inv[6];
                double sy = rx * inv[1] + ry * inv[4] + rz * inv[7];
                double sz = rx * inv[2] + ry * inv[5] + rz * inv[8];
                sx -= rint(sx);
                sy -= rint(sy);
                sz -= rint(sz);
                double dx = sx * lat[0] + sy * lat[3] + sz * lat[6];
                double dy = sx * lat[1] + sy * lat[4] + sz * lat[7];
                double dz = sx * lat[2] + sy * lat[5] + sz * lat[8];
                double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < rl2 && r2 > 1e-20) {
                    if (!count_only) {
                        out_i[n_found] = (int)i;
                        out_j[n_found] = (int)j;
                        out_rij[3 * n_found] = dx;
                        out_rij[3 * n_found + 1] = dy;
                        out_rij[3 * n_found + 2] = dz;
                        out_r[n_found] = sqrt(r2);
                    }
                    ++n_found;
                }
            }
        }
    }
    return n_found;
}

/* ------------------------------------------------------------------ */
/* Tersoff, single species (legacy flat parameters)                     */
/* ------------------------------------------------------------------ */

/* engine/tersoff.py:48-54 */
static double te_fc(double r, double R, double D) {
    if (r < R - D) return 1.0;
    if (r > R + D) return 0.0;
    return 0.5 - 0.5 * sin(0.5 * ORC_PI * (r - R) / D);
}

/* engine/tersoff.py:127-135 */
static double te_dfc(double r, double R, double D) {
    if (r < R - D || r > R + D) return 0.0;
    return -0.25 * ORC_PI / D * cos(0.5 * ORC_PI * (r - R) / D);
}

/* engine/tersoff.py:464-509 (_te_zeta_numpy_par): m = 3 hard-coded, gamma 1. */
void orc_te_zeta(long P, const long *idx_i, const long *idx_j,
                 const double *rij, const double *r,
                 const long *nb_start, const long *nb_idx,
                 const double *nb_rij, const double *nb_r,
                 double *zeta_ij, double *zeta_ji,
                 double l3, double c_t, double d_t, double h_t,
                 double R_t, double D_t)
{
    double l3c = l3 * l3 * l3;
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < P; ++p) {
        long ii = idx_i[p], jj = idx_j[p];
        double r_ij = r[p];
        double zi = 0.0, zj = 0.0;
        for (long nb = nb_start[ii]; nb < nb_start[ii + 1]; ++nb) {
            if (nb_idx[nb] == jj) continue;
            double r_ik = nb_r[nb];
            double fc_ik = te_fc(r_ik, R_t, D_t);
            if (fc_ik == 0.0) continue;
            double dot = 0.0;
            for (int d = 0; d < 3; ++d) dot += rij[3 * p + d] * nb_rij[3 * nb + d];
            double cos_t = dot / (r_ij * r_ik);
            double hc = h_t - cos_t;
            double g_t = 1.0 + c_t * c_t / (d_t * d_t) - c_t * c_t / (d_t * d_t + hc * hc);
            double u = r_ij - r_ik;
            zi += fc_ik * g_t * nb_exp(l3c * (u * u * u));
        }
        for (long nb = nb_start[jj]; nb < nb_start[jj + 1]; ++nb) {
            if (nb_idx[nb] == ii) continue;
            double r_jk = nb_r[nb];
            double fc_jk = te_fc(r_jk, R_t, D_t);
            if (fc_jk == 0.0) continue;
            double dot = 0.0;
            for (int d = 0; d < 3; ++d) dot += (-rij[3 * p + d]) * nb_rij[3 * nb + d];
            double cos_t = dot / (r[p] * r_jk);
            double hc = h_t - cos_t;
            double g_t = 1.0 + c_t * c_t / (d_t * d_t) - c_t * c_t / (d_t * d_t + hc * hc);
            double u = r[p] - r_jk;
            zj += fc_jk * g_t * nb_exp(l3c * (u * u * u));
        }
        zeta_ij[p] += zi;
        zeta_ji[p] += zj;
    }
}

/* engine/tersoff.py:161-202 (_te_zterm_grad): analytic gradient of
 * z = gam fc(r_ik) g(cos) exp(l3^m (r_ij - r_ik)^m) w.r.t. r_ij and r_ik. */
static void te_zterm_grad(double rijx, double rijy, double rijz,
                          double rikx, double riky, double rikz,
                          double R, double D, double c_t, double d_t, double h_t,
                          double l3, double m, double gam, double out[6])
{
    double r_ij = sqrt(rijx * rijx + rijy * rijy + rijz * rijz);
    double r_ik = sqrt(rikx * rikx + riky * riky + rikz * rikz);
    double fc_ik = te_fc(r_ik, R, D);
    if (fc_ik == 0.0) { for (int q = 0; q < 6; ++q) out[q] = 0.0; return; }
    double dfc_ik = te_dfc(r_ik, R, D);
    double inv_ij = 1.0 / r_ij, inv_ik = 1.0 / r_ik;
    double cos_t = (rijx * rikx + rijy * riky + rijz * rikz) * inv_ij * inv_ik;
    double hc = h_t - cos_t;
    double q = d_t * d_t + hc * hc;
    double g_t = 1.0 + c_t * c_t / (d_t * d_t) - c_t * c_t / q;
    double dg = -2.0 * c_t * c_t * hc / (q * q);
    double u = r_ij - r_ik;
    double ex = nb_exp(pow(l3, m) * pow(u, m));
    double dex = ex * m * pow(l3, m) * pow(u, m - 1.0);
    double a_j = gam * fc_ik * dg * ex;
    double b_j = gam * fc_ik * g_t * dex * inv_ij;
    double b_k = gam * (dfc_ik * g_t * ex - fc_ik * g_t * dex) * inv_ik;
    double ii_k = inv_ij * inv_ik;
    double cj = cos_t * inv_ij * inv_ij;
    double ck = cos_t * inv_ik * inv_ik;
    out[0] = a_j * (rikx * ii_k - cj * rijx) + b_j * rijx;
    out[1] = a_j * (riky * ii_k - cj * rijy) + b_j * rijy;
    out[2] = a_j * (rikz * ii_k - cj * rijz) + b_j * rijz;
    out[3] = a_j * (rijx * ii_k - ck * rikx) + b_k * rikx;
    out[4] = a_j * (rijy * ii_k - ck * riky) + b_k * riky;
    out[5] = a_j * (rijz * ii_k - ck * rikz) + b_k * rikz;
}

/* Accumulate one triplet's forces and virial the way engine/tersoff.py:242-275
 * does (center a, partner b, third k; coeff multiplies the zeta gradient). */
static void te_apply(double coeff, const double dz[6], long a, long b, long k,
                     double vbx, double vby, double vbz,
                     double vkx, double vky, double vkz,
                     double *F, double *S)
{
    double Fb0 = -coeff * dz[0], Fb1 = -coeff * dz[1], Fb2 = -coeff * dz[2];
    double Fk0 = -coeff * dz[3], Fk1 = -coeff * dz[4], Fk2 = -coeff * dz[5];
    double Fa0 = coeff * (dz[0] + dz[3]);
    double Fa1 = coeff * (dz[1] + dz[4]);
    double Fa2 = coeff * (dz[2] + dz[5]);
    F[3 * a] += Fa0; F[3 * a + 1] += Fa1; F[3 * a + 2] += Fa2;
    F[3 * b] += Fb0; F[3 * b + 1] += Fb1; F[3 * b + 2] += Fb2;
    F[3 * k] += Fk0; F[3 * k + 1] += Fk1; F[3 * k + 2] += Fk2;
    S[0] += Fb0 * vbx + Fk0 * vkx;
    S[1] += Fb0 * vby + Fk0 * vky;
    S[2] += Fb0 * vbz + Fk0 * vkz;
    S[3] += Fb1 * vbx + Fk1 * vkx;
    S[4] += Fb1 * vby + Fk1 * vky;
    S[5] += Fb1 * vbz + Fk1 * vkz;
    S[6] += Fb2 * vbx + Fk2 * vkx;
    S[7] += Fb2 * vby + Fk2 * vky;
    S[8] += Fb2 * vbz + Fk2 * vkz;
}

/* Sum per-thread buffers into forces/stress (engine/tersoff.py:459-461). */
static void reduce_buffers(int nt, long N, const double *Ft, const double *St,
                           double *forces, double *stress)
{
    for (int t = 0; t < nt; ++t) {
        const double *f = Ft + (size_t)t * N * 3;
        for (long q = 0; q < 3 * N; ++q) forces[q] += f[q];
        for (int q = 0; q < 9; ++q) stress[q] += St[9 * t + q];
    }
}

/* engine/tersoff.py:328-461 (_te_3body_force_numpy_par). */
void orc_te_3body(long p_start, long p_end, long N,
                  const long *idx_i, const long *idx_j,
                  const double *rij, const double *r,
                  const double *fc_arr, const double *fa_arr,
                  const double *dbij_ij, const double *dbij_ji,
                  const long *nb_start, const long *nb_idx,
                  const double *nb_rij, const double *nb_r,
                  double *forces, double *stress,
                  double R, double D, double c_t, double d_t, double h_t,
                  double l3, double m)
{
    int nt = orc_threads();
    double *Ft = calloc((size_t)nt * N * 3, sizeof(double));
    double *St = calloc((size_t)nt * 9, sizeof(double));
    #pragma omp parallel for schedule(static)
    for (long p = p_start; p < p_end; ++p) {
        int tid = orc_tid();
        double *F = Ft + (size_t)tid * N * 3, *S = St + 9 * tid;
        long ii = idx_i[p], jj = idx_j[p];
        double rijx = rij[3 * p], rijy = rij[3 * p + 1], rijz = rij[3 * p + 2];
        double fc_ij = fc_arr[p], fa_ij = fa_arr[p];
        double dbi = dbij_ij[p], dbj = dbij_ji[p];
        double dz[6];
        if (fabs(dbi) > 1e-30) {
            for (long nb = nb_start[ii]; nb < nb_start[ii + 1]; ++nb) {
                long kk = nb_idx[nb];
                if (kk == jj) continue;
                double fc_ik = te_fc(nb_r[nb], R, D);
                if (fc_ik == 0.0) continue;
                double coeff = 0.5 * fc_ij * fa_ij * dbi;
                te_zterm_grad(rijx, rijy, rijz, nb_rij[3 * nb], nb_rij[3 * nb + 1],
                              nb_rij[3 * nb + 2], R, D, c_t, d_t, h_t, l3, m, 1.0, dz);
                te_apply(coeff, dz, ii, jj, kk, rijx, rijy, rijz, nb_rij[3 * nb],
                         nb_rij[3 * nb + 1], nb_rij[3 * nb + 2], F, S);
            }
        }
        if (fabs(dbj) > 1e-30) {
            for (long nb = nb_start[jj]; nb < nb_start[jj + 1]; ++nb) {
                long kk = nb_idx[nb];
                if (kk == ii) continue;
                double fc_jk = te_fc(nb_r[nb], R, D);
                if (fc_jk == 0.0) continue;
                double coeff = 0.5 * fc_ij * fa_ij * dbj;
                te_zterm_grad(-rijx, -rijy, -rijz, nb_rij[3 * nb], nb_rij[3 * nb + 1],
                              nb_rij[3 * nb + 2], R, D, c_t, d_t, h_t, l3, m, 1.0, dz);
                te_apply(coeff, dz, jj, ii, kk, -rijx, -rijy, -rijz, nb_rij[3 * nb],
                         nb_rij[3 * nb + 1], nb_rij[3 * nb + 2], F, S);
            }
        }
    }
    reduce_buffers(nt, N, Ft, St, forces, stress);
    free(Ft);
    free(St);
}

/* ------------------------------------------------------------------ */
/* Tersoff, multi-species (dense species tables)                        */
/* ------------------------------------------------------------------ */

/* Dense tables as engine/tersoff.py:1610-1653 builds them.  tb_* are
 * (ns, ns) row-major, tri_* are (ns, ns, ns) row-major. */
typedef struct {
    long ns;
    const unsigned char *tb_valid;
    const double *tb_A, *tb_B, *tb_l1, *tb_l2, *tb_R, *tb_D;
    const unsigned char *tri_valid;
    const double *tri_c, *tri_d, *tri_h, *tri_l3, *tri_m, *tri_gam;
} orc_te_tables;

/* engine/tersoff.py:609-682 (_te_multi_zeta_numpy_par), including the
 * gating that a pair without a forward (s_i, s_j) entry gets neither zeta. */
void orc_te_multi_zeta(long P, const long *idx_i, const long *idx_j,
                       const double *rij, const double *r, const long *type_ids,
                       const long *nb_start, const long *nb_idx,
                       const double *nb_rij, const double *nb_r,
                       double *zeta_ij, double *zeta_ji, const orc_te_tables *T)
{
    long ns = T->ns;
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < P; ++p) {
        long ii = idx_i[p], jj = idx_j[p];
        long si = type_ids[ii], sj = type_ids[jj];
        if (!T->tb_valid[si * ns + sj]) continue;
        double r_ij = r[p];
        double rijx = rij[3 * p], rijy = rij[3 * p + 1], rijz = rij[3 * p + 2];
        double zi = 0.0, zj = 0.0;
        for (long nb = nb_start[ii]; nb < nb_start[ii + 1]; ++nb) {
            long kk = nb_idx[nb];
            if (kk == jj) continue;
            long sk = type_ids[kk];
            long t3 = (si * ns + sj) * ns + sk;
            if (!T->tb_valid[si * ns + sk] || !T->tri_valid[t3]) continue;
            double r_ik = nb_r[nb];
            double fc_ik = te_fc(r_ik, T->tb_R[si * ns + sk], T->tb_D[si * ns + sk]);
            if (fc_ik == 0.0) continue;
            double dot = rijx * nb_rij[3 * nb] + rijy * nb_rij[3 * nb + 1] + rijz * nb_rij[3 * nb + 2];
            double cos_t = dot / (r_ij * r_ik);
            double c_t = T->tri_c[t3], d_t = T->tri_d[t3], h_t = T->tri_h[t3];
            double hc = h_t - cos_t;
            double g_t = 1.0 + c_t * c_t / (d_t * d_t) - c_t * c_t / (d_t * d_t + hc * hc);
            double mt = T->tri_m[t3];
            zi += T->tri_gam[t3] * fc_ik * g_t * nb_exp(pow(T->tri_l3[t3], mt) * pow(r_ij - r_ik, mt));
        }
        for (long nb = nb_start[jj]; nb < nb_start[jj + 1]; ++nb) {
            long kk = nb_idx[nb];
            if (kk == ii) continue;
            long sk = type_ids[kk];
            long t3 = (sj * ns + si) * ns + sk;
            if (!T->tb_valid[sj * ns + sk] || !T->tri_valid[t3]) continue;
            double r_jk = nb_r[nb];
            double fc_jk = te_fc(r_jk, T->tb_R[sj * ns + sk], T->tb_D[sj * ns + sk]);
            if (fc_jk == 0.0) continue;
            double dot = -rijx * nb_rij[3 * nb] + -rijy * nb_rij[3 * nb + 1] + -rijz * nb_rij[3 * nb + 2];
            double cos_t = dot / (r_ij * r_jk);
            double c_t = T->tri_c[t3], d_t = T->tri_d[t3], h_t = T->tri_h[t3];
            double hc = h_t - cos_t;
            double g_t = 1.0 + c_t * c_t / (d_t * d_t) - c_t * c_t / (d_t * d_t + hc * hc);
            double mt = T->tri_m[t3];
            zj += T->tri_gam[t3] * fc_jk * g_t * nb_exp(pow(T->tri_l3[t3], mt) * pow(r_ij - r_jk, mt));
        }
        zeta_ij[p] += zi;
        zeta_ji[p] += zj;
    }
}

/* engine/tersoff.py:859-1036 (_te_multi_pass3_numpy_par): pair energy and
 * force plus the three-body correction.  Returns the energy. */
double orc_te_multi_pass3(long p_start, long p_end, long N,
                          const long *idx_i, const long *idx_j,
                          const double *rij, const double *r, const long *type_ids,
                          const double *bij_ij, const double *bij_ji,
                          const double *dbij_ij, const double *dbij_ji,
                          const long *nb_start, const long *nb_idx,
                          const double *nb_rij, const double *nb_r,
                          double *forces, double *stress, const orc_te_tables *T)
{
    long ns = T->ns;
    int nt = orc_threads();
    double *Ft = calloc((size_t)nt * N * 3, sizeof(double));
    double *St = calloc((size_t)nt * 9, sizeof(double));
    double energy = 0.0;
    #pragma omp parallel for schedule(static) reduction(+:energy)
    for (long p = p_start; p < p_end; ++p) {
        int tid = orc_tid();
        double *F = Ft + (size_t)tid * N * 3, *S = St + 9 * tid;
        long ii = idx_i[p], jj = idx_j[p];
        long si = type_ids[ii], sj = type_ids[jj];
        long t2 = si * ns + sj;
        if (!T->tb_valid[t2]) continue;
        double A_t = T->tb_A[t2], B_t = T->tb_B[t2], l1 = T->tb_l1[t2], l2 = T->tb_l2[t2];
        double R_t = T->tb_R[t2], D_t = T->tb_D[t2];
        double r_ij = r[p];
        double rijx = rij[3 * p], rijy = rij[3 * p + 1], rijz = rij[3 * p + 2];
        double fc_ij = te_fc(r_ij, R_t, D_t);
        double dfc_ij = te_dfc(r_ij, R_t, D_t);
        if (fc_ij == 0.0 && dfc_ij == 0.0) continue;
        double fr = A_t * nb_exp(-l1 * r_ij);
        double fa = -B_t * nb_exp(-l2 * r_ij);
        double b_avg = 0.5 * (bij_ij[p] + bij_ji[p]);
        energy += fc_ij * (fr + b_avg * fa);
        double dEdr = dfc_ij * (fr + b_avg * fa) + fc_ij * (-l1 * fr + b_avg * (-l2 * fa));
        double cx = dEdr / r_ij;
        double v[3] = {rijx, rijy, rijz};
        for (int d = 0; d < 3; ++d) {
            double fv = cx * v[d];
            F[3 * ii + d] += fv;
            F[3 * jj + d] += -fv;
        }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) S[3 * a + b] -= cx * v[a] * v[b];
        double dbi = dbij_ij[p], dbj = dbij_ji[p];
        double dz[6];
        if (fabs(dbi) > 1e-30) {
            for (long nb = nb_start[ii]; nb < nb_start[ii + 1]; ++nb) {
                long kk = nb_idx[nb];
                if (kk == jj) continue;
                long sk = type_ids[kk];
                long t3 = (si * ns + sj) * ns + sk;
                if (!T->tb_valid[si * ns + sk] || !T->tri_valid[t3]) continue;
                double R_ik = T->tb_R[si * ns + sk], D_ik = T->tb_D[si * ns + sk];
                if (te_fc(nb_r[nb], R_ik, D_ik) == 0.0) continue;
                double coeff = 0.5 * fc_ij * fa * dbi;
                te_zterm_grad(rijx, rijy, rijz, nb_rij[3 * nb], nb_rij[3 * nb + 1], nb_rij[3 * nb + 2],
                              R_ik, D_ik, T->tri_c[t3], T->tri_d[t3], T->tri_h[t3],
                              T->tri_l3[t3], T->tri_m[t3], T->tri_gam[t3], dz);
                te_apply(coeff, dz, ii, jj, kk, rijx, rijy, rijz, nb_rij[3 * nb],
                         nb_rij[3 * nb + 1], nb_rij[3 * nb + 2], F, S);
            }
        }
        if (fabs(dbj) > 1e-30) {
            for (long nb = nb_start[jj]; nb < nb_start[jj + 1]; ++nb) {
                long kk = nb_idx[nb];
                if (kk == ii) continue;
                long sk = type_ids[kk];
                long t3 = (sj * ns + si) * ns + sk;
                if (!T->tb_valid[sj * ns + sk] || !T->tri_valid[t3]) continue;
                double R_jk = T->tb_R[sj * ns + sk], D_jk = T->tb_D[sj * ns + sk];
                if (te_fc(nb_r[nb], R_jk, D_jk) == 0.0) continue;
                double coeff = 0.5 * fc_ij * fa * dbj;
                te_zterm_grad(-rijx, -rijy, -rijz, nb_rij[3 * nb], nb_rij[3 * nb + 1], nb_rij[3 * nb + 2],
                              R_jk, D_jk, T->tri_c[t3], T->tri_d[t3], T->tri_h[t3],
                              T->tri_l3[t3], T->tri_m[t3], T->tri_gam[t3], dz);
                te_apply(coeff, dz, jj, ii, kk, -rijx, -rijy, -rijz, nb_rij[3 * nb],
                         nb_rij[3 * nb + 1], nb_rij[3 * nb + 2], F, S);
            }
        }
    }
    reduce_buffers(nt, N, Ft, St, forces, stress);
    free(Ft);
    free(St);
    return energy;
}

/* ------------------------------------------------------------------ */
/* Stillinger-Weber                                                     */
/* ------------------------------------------------------------------ */

/* engine/stillinger_weber.py:258-306 (_sw_2body_numpy_par). */
double orc_sw_2body(long P, long N, const long *idx_i, const long *idx_j,
                    const double *rij, const double *r,
                    double *forces, double *stress,
                    double eps, double sig, double A_sw, double B_sw,
                    double pp, double qq, double a_sw)
{
    int nt = orc_threads();
    double *Ft = calloc((size_t)nt * N * 3, sizeof(double));
    double *St = calloc((size_t)nt * 9, sizeof(double));
    double energy = 0.0;
    #pragma omp parallel for schedule(static) reduction(+:energy)
    for (long p = 0; p < P; ++p) {
        int tid = orc_tid();
        double *F = Ft + (size_t)tid * N * 3, *S = St + 9 * tid;
        long ii = idx_i[p], jj = idx_j[p];
        double rr = r[p];
        double xi = rr / sig;
        if (xi >= a_sw) continue;
        double t = 1.0 / (xi - a_sw);
        double ex = nb_exp(t);
        double V2 = eps * A_sw * (B_sw * pow(xi, -pp) - pow(xi, -qq)) * ex;
        double dV2 = eps * A_sw * ex * ((-pp * B_sw * pow(xi, -pp - 1) + qq * pow(xi, -qq - 1))
                                        + (B_sw * pow(xi, -pp) - pow(xi, -qq)) * (-t * t));
        double dV2dr = dV2 / sig;
        energy += V2;
        double cx = dV2dr / rr;
        const double *v = rij + 3 * p;
        for (int d = 0; d < 3; ++d) {
            double fv = cx * v[d];
            F[3 * ii + d] += fv;
            F[3 * jj + d] += -fv;
        }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) S[3 * a + b] -= cx * v[a] * v[b];
    }
    reduce_buffers(nt, N, Ft, St, forces, stress);
    free(Ft);
    free(St);
    return energy;
}

/* engine/stillinger_weber.py:96-154 (_sw_h3_grad): h and its gradient
 * w.r.t. r_ij (out[1..3]) and r_ik (out[4..6]). */
static void sw_h3_grad(double rijx, double rijy, double rijz,
                       double rikx, double riky, double rikz,
                       double sig_j, double a_j, double gam_j,
                       double sig_k, double a_k, double gam_k,
                       double c3, double costh0, double out[7])
{
    double r_ij = sqrt(rijx * rijx + rijy * rijy + rijz * rijz);
    double r_ik = sqrt(rikx * rikx + riky * riky + rikz * rikz);
    double xij = r_ij / sig_j, xik = r_ik / sig_k;
    if (xij >= a_j || xik >= a_k) { for (int q = 0; q < 7; ++q) out[q] = 0.0; return; }
    double dj = xij - a_j, dk = xik - a_k;
    double exp_ij = nb_exp(gam_j / dj), exp_ik = nb_exp(gam_k / dk);
    double cos_th = (rijx * rikx + rijy * riky + rijz * rikz) / (r_ij * r_ik);
    double dcos = cos_th - costh0;
    double h = c3 * exp_ij * exp_ik * dcos * dcos;
    double pre = c3 * exp_ij * exp_ik * dcos;
    double inv_ij = 1.0 / r_ij, inv_ik = 1.0 / r_ik;
    double uijx = rijx * inv_ij, uijy = rijy * inv_ij, uijz = rijz * inv_ij;
    double uikx = rikx * inv_ik, uiky = riky * inv_ik, uikz = rikz * inv_ik;
    double rad_j = pre * dcos * (-gam_j / (sig_j * dj * dj));
    double rad_k = pre * dcos * (-gam_k / (sig_k * dk * dk));
    double ang_j = 2.0 * pre * inv_ij, ang_k = 2.0 * pre * inv_ik;
    out[0] = h;
    out[1] = rad_j * uijx + ang_j * (uikx - cos_th * uijx);
    out[2] = rad_j * uijy + ang_j * (uiky - cos_th * uijy);
    out[3] = rad_j * uijz + ang_j * (uikz - cos_th * uijz);
    out[4] = rad_k * uikx + ang_k * (uijx - cos_th * uikx);
    out[5] = rad_k * uiky + ang_k * (uijy - cos_th * uiky);
    out[6] = rad_k * uikz + ang_k * (uijz - cos_th * uikz);
}

static void sw_apply(const double g[7], long i, long j, long k,
                     const double *vj, const double *vk, double *F, double *S)
{
    double fj0 = -g[1], fj1 = -g[2], fj2 = -g[3];
    double fk0 = -g[4], fk1 = -g[5], fk2 = -g[6];
    F[3 * i] += g[1] + g[4]; F[3 * i + 1] += g[2] + g[5]; F[3 * i + 2] += g[3] + g[6];
    F[3 * j] += fj0; F[3 * j + 1] += fj1; F[3 * j + 2] += fj2;
    F[3 * k] += fk0; F[3 * k + 1] += fk1; F[3 * k + 2] += fk2;
    S[0] += fj0 * vj[0] + fk0 * vk[0];
    S[1] += fj0 * vj[1] + fk0 * vk[1];
    S[2] += fj0 * vj[2] + fk0 * vk[2];
    S[3] += fj1 * vj[0] + fk1 * vk[0];
    S[4] += fj1 * vj[1] + fk1 * vk[1];
    S[5] += fj1 * vj[2] + fk1 * vk[2];
    S[6] += fj2 * vj[0] + fk2 * vk[0];
    S[7] += fj2 * vj[1] + fk2 * vk[1];
    S[8] += fj2 * vj[2] + fk2 * vk[2];
}

/* engine/stillinger_weber.py:307-395 (_sw_3body_numpy_par): each unordered
 * neighbour pair (pj < pk) of a centre once. */
double orc_sw_3body(long n_start, long n_end, long N,
                    const long *nb_start, const long *nb_idx,
                    const double *nb_rij, const double *nb_r,
                    double *forces, double *stress,
                    double eps, double sig, double a_sw, double gam,
                    double lam, double costh0)
{
    int nt = orc_threads();
    double *Ft = calloc((size_t)nt * N * 3, sizeof(double));
    double *St = calloc((size_t)nt * 9, sizeof(double));
    double energy = 0.0;
    double c3 = lam * eps;
    #pragma omp parallel for schedule(static) reduction(+:energy)
    for (long i = n_start; i < n_end; ++i) {
        int tid = orc_tid();
        double *F = Ft + (size_t)tid * N * 3, *S = St + 9 * tid;
        long si = nb_start[i], ei = nb_start[i + 1];
        if (ei - si < 2) continue;
        for (long pj = si; pj < ei; ++pj) {
            if (nb_r[pj] / sig >= a_sw) continue;
            for (long pk = pj + 1; pk < ei; ++pk) {
                if (nb_r[pk] / sig >= a_sw) continue;
                double g[7];
                const double *vj = nb_rij + 3 * pj, *vk = nb_rij + 3 * pk;
                sw_h3_grad(vj[0], vj[1], vj[2], vk[0], vk[1], vk[2],
                           sig, a_sw, gam, sig, a_sw, gam, c3, costh0, g);
                energy += g[0];
                sw_apply(g, i, nb_idx[pj], nb_idx[pk], vj, vk, F, S);
            }
        }
    }
    reduce_buffers(nt, N, Ft, St, forces, stress);
    free(Ft);
    free(St);
    return energy;
}

/* engine/stillinger_weber.py:414-453 (_sw_multi_2body_numpy), serial. */
double orc_sw_multi_2body(long P, long N, const long *idx_i, const long *idx_j,
                          const double *rij, const double *r, const long *type_ids,
                          double *forces, double *stress, long ns,
                          const unsigned char *tb_valid, const double *tb_eps,
                          const double *tb_sig, const double *tb_a, const double *tb_A,
                          const double *tb_B, const double *tb_p, const double *tb_q)
{
    double energy = 0.0;
    for (long p = 0; p < P; ++p) {
        long ii = idx_i[p], jj = idx_j[p];
        long t2 = type_ids[ii] * ns + type_ids[jj];
        if (!tb_valid[t2]) continue;
        double sig = tb_sig[t2], a_sw = tb_a[t2];
        double rr = r[p];
        double xi = rr / sig;
        if (xi >= a_sw) continue;
        double eps = tb_eps[t2], A_sw = tb_A[t2], B_sw = tb_B[t2];
        double pp = tb_p[t2], qq = tb_q[t2];
        double t = 1.0 / (xi - a_sw);
        double ex = nb_exp(t);
        double V2 = eps * A_sw * (B_sw * pow(xi, -pp) - pow(xi, -qq)) * ex;
        double dV2 = eps * A_sw * ex * ((-pp * B_sw * pow(xi, -pp - 1) + qq * pow(xi, -qq - 1))
                                        + (B_sw * pow(xi, -pp) - pow(xi, -qq)) * (-t * t));
        double dV2dr = dV2 / sig;
        energy += V2;
        double cx = dV2dr / rr;
        const double *v = rij + 3 * p;
        for (int d = 0; d < 3; ++d) {
            double fv = cx * v[d];
            forces[3 * ii + d] += fv;
            forces[3 * jj + d] += -fv;
        }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) stress[3 * a + b] -= cx * v[a] * v[b];
    }
    return energy;
}

/* engine/stillinger_weber.py:570-662 (_sw_multi_3body_numpy_par): both
 * orders (j, k) and (k, j), each with lambda/2 of its own record. */
double orc_sw_multi_3body(long n_start, long n_end, long N,
                          const long *nb_start, const long *nb_idx,
                          const double *nb_rij, const double *nb_r, const long *type_ids,
                          double *forces, double *stress, long ns,
                          const unsigned char *tri_valid, const double *tri_eps,
                          const double *tri_lam, const double *tri_cos,
                          const double *leg_sig, const double *leg_a, const double *leg_gam)
{
    (void)nb_r;
    int nt = orc_threads();
    double *Ft = calloc((size_t)nt * N * 3, sizeof(double));
    double *St = calloc((size_t)nt * 9, sizeof(double));
    double energy = 0.0;
    #pragma omp parallel for schedule(static) reduction(+:energy)
    for (long i = n_start; i < n_end; ++i) {
        int tid = orc_tid();
        double *F = Ft + (size_t)tid * N * 3, *S = St + 9 * tid;
        long si = nb_start[i], ei = nb_start[i + 1];
        if (ei - si < 2) continue;
        long i_sp = type_ids[i];
        for (long pj = si; pj < ei; ++pj) {
            long j_at = nb_idx[pj], j_sp = type_ids[j_at];
            const double *vj = nb_rij + 3 * pj;
            for (long pk = si; pk < ei; ++pk) {
                if (pk == pj) continue;
                long k_at = nb_idx[pk], k_sp = type_ids[k_at];
                long t3 = (i_sp * ns + j_sp) * ns + k_sp;
                if (!tri_valid[t3]) continue;
                const double *vk = nb_rij + 3 * pk;
                long lj = i_sp * ns + j_sp, lk = i_sp * ns + k_sp;
                double lam_t = 0.5 * tri_lam[t3];
                double g[7];
                sw_h3_grad(vj[0], vj[1], vj[2], vk[0], vk[1], vk[2],
                           leg_sig[lj], leg_a[lj], leg_gam[lj],
                           leg_sig[lk], leg_a[lk], leg_gam[lk],
                           tri_eps[t3] * lam_t, tri_cos[t3], g);
                if (g[0] == 0.0) continue;
                energy += g[0];
                sw_apply(g, i, j_at, k_at, vj, vk, F, S);
            }
        }
    }
    reduce_buffers(nt, N, Ft, St, forces, stress);
    free(Ft);
    free(St);
    return energy;
}

/* ------------------------------------------------------------------ */
/* EAM                                                                  */
/* ------------------------------------------------------------------ */

/* function codes and parameter slots of engine/_eam_kernels.py:30-60 */
enum { F_SPLINE = 1, F_SPLINE_R = 2, F_Z_DENS = 3, F_Z_PAIR = 4, F_Z_CROSS = 5, F_Z_EMB = 6 };
#define NZ 20

typedef struct {
    const long *codes;
    const double *P;     /* (nf, ncol) */
    long ncol;
    const long *xo, *nx;
    const double *X;     /* (nX,) */
    const double *C;     /* (4, nX) */
    long nX;
} orc_eam_tables;

/* engine/_eam_kernels.py:129-145 (_spline_eval): scipy's interval choice
 * (searchsorted side='right' - 1, clipped to the end intervals) and Horner. */
static void spline_eval(const orc_eam_tables *T, long o, long n, double r,
                        double *v, double *dv)
{
    long lo = 0, hi = n;
    while (lo < hi) {
        long mid = (lo + hi) / 2;
        if (T->X[o + mid] <= r) lo = mid + 1; else hi = mid;
    }
    long i = lo - 1;
    if (i < 0) i = 0;
    if (i > n - 2) i = n - 2;
    double dx = r - T->X[o + i];
    double c0 = T->C[o + i], c1 = T->C[T->nX + o + i];
    double c2 = T->C[2 * T->nX + o + i], c3 = T->C[3 * T->nX + o + i];
    *v = ((c0 * dx + c1) * dx + c2) * dx + c3;
    *dv = (3.0 * c0 * dx + 2.0 * c1) * dx + c2;
}

/* engine/_eam_kernels.py:148-155 (_decay) */
static void decay(double r, double re, double pre, double expo, double shift,
                  double *val, double *dval)
{
    double x = r / re;
    double e = pre * exp(-expo * (x - 1.0));
    double u = x - shift;
    double u2 = u * u, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8;
    double u19 = u16 * u2 * u;
    double u20 = u16 * u4;
    double den = 1.0 + u20;
    *val = e / den;
    *dval = (-expo * e / den - e * 20.0 * u19 / (den * den)) / re;
}

static void zdens(const double *p, double r, double *v, double *dv)
{
    decay(r, p[0], p[1], p[5], p[9], v, dv);
}

static void zpair(const double *p, double r, double *v, double *dv)
{
    double a, da, b, db;
    decay(r, p[0], p[6], p[4], p[8], &a, &da);
    decay(r, p[0], p[7], p[5], p[9], &b, &db);
    *v = a - b;
    *dv = da - db;
}

/* engine/_eam_kernels.py:170-177 (_switch) */
static void zswitch(double r, double rc, double w, double *S, double *dS)
{
    double s = (r - (rc - w)) / w;
    if (s < 0.0) s = 0.0; else if (s > 1.0) s = 1.0;
    *S = 1.0 - s * s * s * (10.0 - 15.0 * s + 6.0 * s * s);
    *dS = -30.0 * s * s * (1.0 - s) * (1.0 - s) / w;
}

/* engine/_eam_kernels.py:180-196 (_embed) */
static void zembed(const double *p, double rho, double *F, double *dF)
{
    double re = p[2], rs = p[3], eta = p[18];
    double rn = 0.85 * re;
    if (rho < rn) {
        double z = rho / rn - 1.0;
        *F = p[10] + p[11] * z + p[12] * z * z + p[13] * z * z * z;
        *dF = (p[11] + 2 * p[12] * z + 3 * p[13] * z * z) / rn;
    } else if (rho >= 1.15 * re) {
        double t = rho / rs;
        double lt = log(t);
        *F = p[19] * (1.0 - eta * lt) * pow(t, eta);
        *dF = -p[19] * eta * eta * lt * pow(t, eta - 1.0) / rs;
    } else {
        double z = rho / re - 1.0;
        *F = p[14] + p[15] * z + p[16] * z * z + p[17] * z * z * z;
        *dF = (p[15] + 2 * p[16] * z + 3 * p[17] * z * z) / re;
    }
}

/* engine/_eam_kernels.py:199-228 (_feval) */
static void feval(const orc_eam_tables *T, long f, double r, double *v, double *dv)
{
    long code = T->codes[f];
    const double *P = T->P + f * T->ncol;
    if (code == F_SPLINE) { spline_eval(T, T->xo[f], T->nx[f], r, v, dv); return; }
    if (code == F_SPLINE_R) {
        double s, ds;
        spline_eval(T, T->xo[f], T->nx[f], r, &s, &ds);
        *v = s / r;
        *dv = (ds * r - s) / (r * r);
        return;
    }
    if (code == F_Z_EMB) { zembed(P, r, v, dv); return; }
    double val, dval;
    if (code == F_Z_DENS) {
        zdens(P, r, &val, &dval);
    } else if (code == F_Z_PAIR) {
        zpair(P, r, &val, &dval);
    } else {
        double fa, dfa, fb, dfb, ua, dua, ub, dub;
        zdens(P, r, &fa, &dfa);
        zdens(P + NZ, r, &fb, &dfb);
        zpair(P, r, &ua, &dua);
        zpair(P + NZ, r, &ub, &dub);
        double k = P[2 * NZ + 2];
        double q = fb / fa;
        double dq = (dfb * fa - fb * dfa) / (fa * fa);
        val = 0.5 * k * (q * ua + ub / q);
        dval = 0.5 * k * (dq * ua + q * dua + dub / q - ub * dq / (q * q));
    }
    double S, dS;
    zswitch(r, P[2 * NZ], P[2 * NZ + 1], &S, &dS);
    *v = val * S;
    *dv = dval * S + val * dS;
}

/* engine/_eam_kernels.py:231-307 (_eam_kernel): energy, forces and the
 * virial sum -sum f (x) r (not yet divided by the volume). */
double orc_eam_kernel(long N, long npair, const long *ii, const long *jj,
                      const double *rij, const double *r, const long *spc,
                      const long *RHO, const long *FF, const long *PHI, long ns,
                      const orc_eam_tables *T, double *forces, double *vir)
{
    double *rho_i = malloc(sizeof(double) * npair), *drho_j = malloc(sizeof(double) * npair);
    double *rho_j = malloc(sizeof(double) * npair), *drho_i = malloc(sizeof(double) * npair);
    double *phi = malloc(sizeof(double) * npair), *dphi = malloc(sizeof(double) * npair);
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < npair; ++p) {
        long si = spc[ii[p]], sj = spc[jj[p]];
        feval(T, RHO[sj], r[p], &rho_i[p], &drho_j[p]);
        feval(T, RHO[si], r[p], &rho_j[p], &drho_i[p]);
        feval(T, PHI[si * ns + sj], r[p], &phi[p], &dphi[p]);
    }
    long *cnt = calloc(N + 1, sizeof(long));
    for (long p = 0; p < npair; ++p) { cnt[ii[p] + 1] += 1; cnt[jj[p] + 1] += 1; }
    for (long a = 0; a < N; ++a) cnt[a + 1] += cnt[a];
    long *fill = malloc(sizeof(long) * (N + 1));
    memcpy(fill, cnt, sizeof(long) * N);
    long *lst = malloc(sizeof(long) * 2 * npair);
    long *side = malloc(sizeof(long) * 2 * npair);
    for (long p = 0; p < npair; ++p) {
        long a = ii[p];
        lst[fill[a]] = p; side[fill[a]] = 1; fill[a] += 1;
        long b = jj[p];
        lst[fill[b]] = p; side[fill[b]] = -1; fill[b] += 1;
    }
    double *Fv = malloc(sizeof(double) * N), *dF = malloc(sizeof(double) * N);
    #pragma omp parallel for schedule(static)
    for (long a = 0; a < N; ++a) {
        double rb = 0.0;
        for (long k = cnt[a]; k < cnt[a + 1]; ++k) {
            long p = lst[k];
            rb += side[k] == 1 ? rho_i[p] : rho_j[p];
        }
        if (rb < 0.0) rb = 0.0;
        feval(T, FF[spc[a]], rb, &Fv[a], &dF[a]);
    }
    double *fij = malloc(sizeof(double) * 3 * npair);
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < npair; ++p) {
        double c = dphi[p] + dF[ii[p]] * drho_j[p] + dF[jj[p]] * drho_i[p];
        double s = c / r[p];
        fij[3 * p] = s * rij[3 * p];
        fij[3 * p + 1] = s * rij[3 * p + 1];
        fij[3 * p + 2] = s * rij[3 * p + 2];
    }
    #pragma omp parallel for schedule(static)
    for (long a = 0; a < N; ++a) {
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (long k = cnt[a]; k < cnt[a + 1]; ++k) {
            long p = lst[k];
            double sg = (double)side[k];
            fx += sg * fij[3 * p];
            fy += sg * fij[3 * p + 1];
            fz += sg * fij[3 * p + 2];
        }
        forces[3 * a] = fx; forces[3 * a + 1] = fy; forces[3 * a + 2] = fz;
    }
    for (int q = 0; q < 9; ++q) vir[q] = 0.0;
    for (long p = 0; p < npair; ++p)
        for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 3; ++y) vir[3 * x + y] -= fij[3 * p + x] * rij[3 * p + y];
    double energy = 0.0;
    for (long a = 0; a < N; ++a) energy += Fv[a];
    double ephi = 0.0;
    for (long p = 0; p < npair; ++p) ephi += phi[p];
    free(rho_i); free(drho_j); free(rho_j); free(drho_i); free(phi); free(dphi);
    free(cnt); free(fill); free(lst); free(side); free(Fv); free(dF); free(fij);
    return energy + ephi;
}
