// Alloy EAM: density kernel (rho-bar, F, F') and force kernel, lane group
// per atom over the two-way CSR, no atomics.
//
// Replaces engine/eam.py:174-256 and engine/_eam_kernels.py:231-307.  The
// reference evaluates each half pair once and scatters through a serial
// two-way CSR; here each atom gathers over its own row (owner computes), so
// a pair's functions are evaluated from both sides and nothing is written
// twice.  rho-bar is accumulated and clamped in float64 and F(rho-bar) is
// evaluated in float64 in both precisions.
#include <mutex>

#include "mbf_util.cuh"

namespace mbf {

constexpr int EAM_NZ = 20;         // Zhou parameters per element row
constexpr int EAM_NCOL = 2 * EAM_NZ + 3;
constexpr int EAM_MAXSP = 8;       // species staged in shared memory (fused path)
constexpr int EAM_BLOCK = 128;
// Resident blocks per SM the float32 force kernel is compiled for (it sets
// the register budget: 65536 / (EAM_BLOCK * MBF_EAM_MINB)).
#ifndef MBF_EAM_MINB
#define MBF_EAM_MINB 5
#endif
// The same for the float32 density kernel (48 registers, no spills).
#ifndef MBF_EAM_DENS_MINB
#define MBF_EAM_DENS_MINB 10
#endif

enum { F_SPLINE = 1, F_SPLINE_R = 2, F_Z_DENS = 3, F_Z_PAIR = 4, F_Z_CROSS = 5, F_Z_EMB = 6 };

struct EamDev {
    int ns, nf, nX;
    const int *codes;
    const double *P;
    const int *xo, *nx;
    const double *X, *C;
    const int *rho_f, *F_f, *phi_f;
    double r_cut;
};

// Bounds checks on every neighbour-list index the kernels dereference: a
// failed check records (site, index) in the workspace error words and skips
// the access; mbf_eval_status() returns them to the host.  They are always
// compiled in: the float64 build of these kernels without them raised an
// illegal-address fault on B200 whose cause was not found, while the checked
// build, with the same indices, runs clean.
// Every index and bound is an int (the entries refuse lists of more than
// 0x7fffff00 slots, so a slot index plus its prefetch distance cannot
// overflow), so lo <= idx < hi is one unsigned comparison: idx - lo taken
// modulo 2^32 is below hi - lo exactly when idx is in range.
struct Chk {
    int *err;
    int n_atoms;
    int n_slots;
    int ns;
};
#define MBF_OK_IDX(ck, site, idx, lo, hi)                                                          \
    (((unsigned)(int)(idx) - (unsigned)(int)(lo) < (unsigned)max((int)(hi) - (int)(lo), 0))       \
         ? true                                                                                    \
         : (atomicCAS((ck).err + 1, 0, (site)) == 0 ? ((ck).err[2] = (int)(idx), false) : false))

// ---- generic function evaluation (engine/_eam_kernels.py:129-228) -------

template <typename T>
__device__ __forceinline__ void spline_eval(const EamDev &E, int f, double r, T &v, T &dv) {
    int o = E.xo[f], n = E.nx[f];
    const double *X = E.X + o;
    const double *Pf = E.P + (size_t)f * EAM_NCOL;
    int i;
    if (Pf[0] == 1.0) {
        // uniform knots: the interval from the spacing, then moved by at most
        // one so that it is the last knot <= r, as the search below gives
        double t = (r - Pf[1]) * Pf[2];
        int k = t < 0.0 ? 0 : (t > (double)(n - 1) ? n - 1 : (int)t);
        if (k + 1 < n && X[k + 1] <= r) ++k;
        else if (k > 0 && X[k] > r) --k;
        i = k;
    } else {
        int lo = 0, hi = n;
        while (lo < hi) {  // searchsorted(side='right')
            int mid = (lo + hi) >> 1;
            if (X[mid] <= r) lo = mid + 1; else hi = mid;
        }
        i = lo - 1;
    }
    i = i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
    T dx = (T)(r - X[i]);
    T c0 = (T)E.C[o + i], c1 = (T)E.C[E.nX + o + i];
    T c2 = (T)E.C[2 * E.nX + o + i], c3 = (T)E.C[3 * E.nX + o + i];
    v = ((c0 * dx + c1) * dx + c2) * dx + c3;
    dv = (T(3) * c0 * dx + T(2) * c1) * dx + c2;
}

template <typename T>
__device__ __forceinline__ void zdecay(T r, T re, T pre, T expo, T shift, T &val, T &dval) {
    T x = r / re;
    T e = pre * RT<T>::ex(-expo * (x - T(1)));
    T u19;
    T den = T(1) + pow20(x - shift, u19);
    val = e / den;
    dval = (-expo * e / den - e * T(20) * u19 / (den * den)) / re;
}

template <typename T>
__device__ __forceinline__ void zdens(const double *p, T r, T &v, T &dv) {
    zdecay<T>(r, (T)p[0], (T)p[1], (T)p[5], (T)p[9], v, dv);
}

template <typename T>
__device__ __forceinline__ void zpair(const double *p, T r, T &v, T &dv) {
    T a, da, b, db;
    zdecay<T>(r, (T)p[0], (T)p[6], (T)p[4], (T)p[8], a, da);
    zdecay<T>(r, (T)p[0], (T)p[7], (T)p[5], (T)p[9], b, db);
    v = a - b;
    dv = da - db;
}

template <typename T>
__device__ __forceinline__ void zswitch(T r, T rc, T w, T &S, T &dS) {
    T s = (r - (rc - w)) / w;
    s = s < T(0) ? T(0) : (s > T(1) ? T(1) : s);
    S = T(1) - s * s * s * (T(10) - T(15) * s + T(6) * s * s);
    dS = T(-30) * s * s * (T(1) - s) * (T(1) - s) / w;
}

// Zhou embedding, eqs. (A6)-(A8) (engine/_eam_kernels.py:180-196); float64.
__device__ __forceinline__ void zembed(const double *p, double rho, double &F, double &dF) {
    double re = p[2], rs = p[3], eta = p[18];
    double rn = 0.85 * re;
    if (rho < rn) {
        double z = rho / rn - 1.0;
        F = p[10] + p[11] * z + p[12] * z * z + p[13] * z * z * z;
        dF = (p[11] + 2 * p[12] * z + 3 * p[13] * z * z) / rn;
    } else if (rho >= 1.15 * re) {
        double t = rho / rs;
        double lt = log(t);
        F = p[19] * (1.0 - eta * lt) * pow(t, eta);
        dF = -p[19] * eta * eta * lt * pow(t, eta - 1.0) / rs;
    } else {
        double z = rho / re - 1.0;
        F = p[14] + p[15] * z + p[16] * z * z + p[17] * z * z * z;
        dF = (p[15] + 2 * p[16] * z + 3 * p[17] * z * z) / re;
    }
}

template <typename T>
__device__ void feval(const EamDev &E, int f, double r, T &v, T &dv) {
    int code = E.codes[f];
    const double *P = E.P + (size_t)f * EAM_NCOL;
    if (code == F_SPLINE) {
        spline_eval<T>(E, f, r, v, dv);
        return;
    }
    if (code == F_SPLINE_R) {
        T s, ds;
        spline_eval<T>(E, f, r, s, ds);
        T rr = (T)r;
        v = s / rr;
        dv = (ds * rr - s) / (rr * rr);
        return;
    }
    if (code == F_Z_EMB) {
        double F, dF;
        zembed(P, r, F, dF);
        v = (T)F;
        dv = (T)dF;
        return;
    }
    T rr = (T)r, val, dval;
    if (code == F_Z_DENS) {
        zdens<T>(P, rr, val, dval);
    } else if (code == F_Z_PAIR) {
        zpair<T>(P, rr, val, dval);
    } else {
        T fa, dfa, fb, dfb, ua, dua, ub, dub;
        zdens<T>(P, rr, fa, dfa);
        zdens<T>(P + EAM_NZ, rr, fb, dfb);
        zpair<T>(P, rr, ua, dua);
        zpair<T>(P + EAM_NZ, rr, ub, dub);
        T k = (T)P[2 * EAM_NZ + 2];
        T q = fb / fa;
        T dq = (dfb * fa - fb * dfa) / (fa * fa);
        val = T(0.5) * k * (q * ua + ub / q);
        dval = T(0.5) * k * (dq * ua + q * dua + dub / q - ub * dq / (q * q));
    }
    T S, dS;
    zswitch<T>(rr, (T)P[2 * EAM_NZ], (T)P[2 * EAM_NZ + 1], S, dS);
    v = val * S;
    dv = dval * S + val * dS;
}

// Embedding F(rho) always in float64.
__device__ __forceinline__ void embed64(const EamDev &E, int f, double rho, double &F, double &dF) {
    if (E.codes[f] == F_Z_EMB) {
        zembed(E.P + (size_t)f * EAM_NCOL, rho, F, dF);
    } else {
        feval<double>(E, f, rho, F, dF);
    }
}

// ---- fused Zhou alloy path ----------------------------------------------
// One element's density f and pair phi_aa share exp(-beta (x - 1)) and the
// denominator 1 + (x - lambda)^20, so a species costs two exponentials.

template <typename T>
struct ZSp {
    T inv_re, fe, beta, lam, A, alpha, kappa, B;
};

template <typename T>
struct ZTab {
    ZSp<T> sp[EAM_MAXSP];
    T chi[EAM_MAXSP * EAM_MAXSP];
    T rc, w, inv_w;
};

template <typename T>
__device__ __forceinline__ void zspecies(const ZSp<T> &p, T r, T &f, T &df, T &pr, T &dpr) {
    T x = r * p.inv_re;
    T xm1 = x - T(1);
    T eB = RT<T>::ex(-p.beta * xm1);
    T eA = RT<T>::ex(-p.alpha * xm1);
    T u19B, u19A;
    T rdB = fdiv<T>(T(1), T(1) + pow20(x - p.lam, u19B));
    T rdA = fdiv<T>(T(1), T(1) + pow20(x - p.kappa, u19A));
    T gB = eB * rdB, gA = eA * rdA;
    T dgB = gB * (-p.beta - T(20) * u19B * rdB);
    T dgA = gA * (-p.alpha - T(20) * u19A * rdA);
    f = p.fe * gB;
    df = p.fe * dgB * p.inv_re;
    pr = p.A * gA - p.B * gB;
    dpr = (p.A * dgA - p.B * dgB) * p.inv_re;
}

template <typename T>
__device__ __forceinline__ T zdens_only(const ZSp<T> &p, T r) {
    T x = r * p.inv_re;
    T u19;
    T d = T(1) + pow20(x - p.lam, u19);
    return fdiv<T>(p.fe * RT<T>::ex(-p.beta * (x - T(1))), d);
}

template <typename T>
__device__ __forceinline__ void zswitch_fast(T r, const ZTab<T> &Z, T &S, T &dS) {
    T s = (r - (Z.rc - Z.w)) * Z.inv_w;
    s = s < T(0) ? T(0) : (s > T(1) ? T(1) : s);
    S = T(1) - s * s * s * (T(10) - T(15) * s + T(6) * s * s);
    dS = T(-30) * s * s * (T(1) - s) * (T(1) - s) * Z.inv_w;
}

template <typename T>
__device__ void load_ztab(const EamDev &E, ZTab<T> &Z) {
    for (int s = threadIdx.x; s < E.ns; s += blockDim.x) {
        const double *p = E.P + (size_t)E.rho_f[s] * EAM_NCOL;
        ZSp<T> q;
        q.inv_re = (T)(1.0 / p[0]); q.fe = (T)p[1]; q.beta = (T)p[5]; q.lam = (T)p[9];
        q.A = (T)p[6]; q.alpha = (T)p[4]; q.kappa = (T)p[8]; q.B = (T)p[7];
        Z.sp[s] = q;
    }
    for (int ab = threadIdx.x; ab < E.ns * E.ns; ab += blockDim.x) {
        int a = ab / E.ns, b = ab % E.ns;
        T k = T(1);
        if (a != b) k = (T)E.P[(size_t)E.phi_f[a * E.ns + b] * EAM_NCOL + 2 * EAM_NZ + 2];
        Z.chi[a * EAM_MAXSP + b] = k;
    }
    if (threadIdx.x == 0) {
        const double *p = E.P + (size_t)E.rho_f[0] * EAM_NCOL;
        Z.rc = (T)p[2 * EAM_NZ];
        Z.w = (T)p[2 * EAM_NZ + 1];
        Z.inv_w = (T)(1.0 / p[2 * EAM_NZ + 1]);
    }
    __syncthreads();
}

// phi_{si,sj}, rho'_{sj}, rho'_{si} at r (fused Zhou path).
// phi_{si,sj}, rho'_{sj}, rho'_{si} at r (fused Zhou path), without a
// branch on the species: both species' functions are evaluated and combined
// by the cross-pair rule phi_ab = 1/2 k (q phi_aa + phi_bb / q), q = f_b/f_a
// (engine/eam_zhou.py:128-207), which for a == b (k = 1, q = 1) is phi_aa
// up to rounding -- so the lanes of a warp never split between the like and
// the cross path of a random alloy.
template <typename T>
__device__ __forceinline__ void zhou_pair_terms(const ZTab<T> &Z, int si, int sj, T r, T &phi,
                                                T &dphi, T &drho_j, T &drho_i) {
    T S, dS;
    zswitch_fast<T>(r, Z, S, dS);
    int a = min(si, sj), b = max(si, sj);
    T fa, dfa, ua, dua, fb, dfb, ub, dub;
    zspecies<T>(Z.sp[a], r, fa, dfa, ua, dua);
    zspecies<T>(Z.sp[b], r, fb, dfb, ub, dub);
    T k = Z.chi[a * EAM_MAXSP + b];
    T rfa = fdiv<T>(T(1), fa);
    T q = fb * rfa;
    T rq = fdiv<T>(T(1), q);
    T dq = (dfb * fa - fb * dfa) * rfa * rfa;
    T v = T(0.5) * k * (q * ua + ub * rq);
    T dv = T(0.5) * k * (dq * ua + q * dua + dub * rq - ub * dq * rq * rq);
    phi = v * S;
    dphi = dv * S + v * dS;
    T dra = dfa * S + fa * dS, drb = dfb * S + fb * dS;
    drho_j = sj == a ? dra : drb;
    drho_i = si == a ? dra : drb;
}

// Minimum image for the force kernels (fused multiply-add allowed).
__device__ __forceinline__ void mic_fast(const double *__restrict__ c, double rx, double ry, double rz,
                                         double &dx, double &dy, double &dz) {
    double sx = rx * c[9] + ry * c[12] + rz * c[15];
    double sy = rx * c[10] + ry * c[13] + rz * c[16];
    double sz = rx * c[11] + ry * c[14] + rz * c[17];
    sx -= rint_shift(sx);
    sy -= rint_shift(sy);
    sz -= rint_shift(sz);
    dx = sx * c[0] + sy * c[3] + sz * c[6];
    dy = sx * c[1] + sy * c[4] + sz * c[7];
    dz = sx * c[2] + sy * c[5] + sz * c[8];
}

// The cell of one atom as the force kernels need it: a diagonal cell keeps
// six scalars (lengths and inverse lengths) instead of the 3x3 pair.
template <bool ORTHO>
struct CellView {
    const double *c;
    double L0, L1, L2, i0, i1, i2;
    __device__ __forceinline__ void load(const SysView &S, int atom) {
        c = cell_of(S, atom);
        if (ORTHO) {
            L0 = c[0]; L1 = c[4]; L2 = c[8];
            i0 = c[9]; i1 = c[13]; i2 = c[17];
        }
    }
    __device__ __forceinline__ void mic(double rx, double ry, double rz, double &dx, double &dy,
                                        double &dz) const {
        if (ORTHO) {
            dx = rx - L0 * rint_shift(rx * i0);
            dy = ry - L1 * rint_shift(ry * i1);
            dz = rz - L2 * rint_shift(rz * i2);
        } else {
            mic_fast(c, rx, ry, rz, dx, dy, dz);
        }
    }
};

// Distance of a minimum-imaged displacement in the working precision: the
// wrap and the square stay float64; the root is taken in T.
template <typename T>
__device__ __forceinline__ T pair_dist(double r2);
template <> __device__ __forceinline__ double pair_dist<double>(double r2) { return sqrt(r2); }
template <> __device__ __forceinline__ float pair_dist<float>(double r2) { return sqrtf((float)r2); }

// ---- kernels --------------------------------------------------------------

// Per-atom record read by every neighbour: position and, once the density
// pass has run, F'(rho-bar) -- one 32-byte sector per neighbour gather.
__global__ void eam_pack(SysView S, double4 *__restrict__ pk) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n_atoms) return;
    pk[i] = make_double4(S.pos[3 * (size_t)i], S.pos[3 * (size_t)i + 1], S.pos[3 * (size_t)i + 2], 0.0);
}

__device__ __forceinline__ double4 ld_pack(const double4 *__restrict__ pk, int j) {
    const double2 *p = reinterpret_cast<const double2 *>(pk + j);
    double2 a = __ldg(p), b = __ldg(p + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// rho-bar_i over the full row, F(rho-bar_i) and F'(rho-bar_i) in float64.
// The next neighbour's index, record and species are loaded one iteration
// ahead of their use.
template <typename T, int LPA, bool ZHOU, bool ORTHO>
__global__ void __launch_bounds__(EAM_BLOCK, sizeof(T) == 4 ? MBF_EAM_DENS_MINB : 1) eam_density(SysView S, const int *__restrict__ row_off,
                                                         const int *__restrict__ nbr, EamDev E,
                                                         double4 *__restrict__ pk,
                                                         double *__restrict__ aux, Chk ck) {
    __shared__ ZTab<T> Z;
    if (ZHOU) load_ztab<T>(E, Z);
    const int sub = threadIdx.x & (LPA - 1);
    const int gpb = EAM_BLOCK / LPA;
    const double rc = E.r_cut, rc2 = rc * rc;
    for (int base = blockIdx.x * gpb; base < S.n_atoms; base += gridDim.x * gpb) {
        int i = base + threadIdx.x / LPA;
        double acc = 0.0;
        if (i < S.n_atoms) {
            CellView<ORTHO> cv;
            cv.load(S, i);
            double4 pi = ld_pack(pk, i);
            int end = row_off[i + 1];
            int s = row_off[i] + sub;
            if (!MBF_OK_IDX(ck, 11, end, 0, ck.n_slots + 1)) end = s;
            // two-stage prefetch, as in eam_force
            int j0 = i, j1 = i;
            if (s < end && MBF_OK_IDX(ck, 12, s, 0, ck.n_slots)) j0 = nbr[s];
            if (s + LPA < end && MBF_OK_IDX(ck, 15, s + LPA, 0, ck.n_slots)) j1 = nbr[s + LPA];
            if (!MBF_OK_IDX(ck, 13, j0, 0, ck.n_atoms)) j0 = i;
            double4 pn = ld_pack(pk, j0);
            int tn = __ldg(S.types + j0);
            for (; s < end; s += LPA) {
                double4 pj = pn;
                int sj = tn;
                if (!MBF_OK_IDX(ck, 14, sj, 0, ck.ns)) sj = 0;
                if (s + LPA < end) {
                    if (!MBF_OK_IDX(ck, 16, j1, 0, ck.n_atoms)) j1 = i;
                    pn = ld_pack(pk, j1);
                    tn = __ldg(S.types + j1);
                }
                if (s + 2 * LPA < end && MBF_OK_IDX(ck, 15, s + 2 * LPA, 0, ck.n_slots)) j1 = nbr[s + 2 * LPA];
                double dx, dy, dz;
                cv.mic(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z, dx, dy, dz);
                double r2 = dx * dx + dy * dy + dz * dz;
                if (!(r2 < rc2 && r2 > 1e-24)) continue;
                if (ZHOU) {
                    T r = pair_dist<T>(r2);
                    T Sw, dSw;
                    zswitch_fast<T>(r, Z, Sw, dSw);
                    acc += (double)(zdens_only<T>(Z.sp[sj], r) * Sw);
                } else {
                    T v, dv;
                    feval<T>(E, E.rho_f[sj], sqrt(r2), v, dv);
                    acc += (double)v;
                }
            }
        }
        acc = group_sum<LPA>(acc);
        if (sub == 0 && i < S.n_atoms) aux[2 * (size_t)i] = acc;
    }
}

// F(rho-bar) and F'(rho-bar) in float64, rho-bar clamped at 0
// (engine/_eam_kernels.py:268-274); kept out of the density loop so the
// float64 pow/log of the embedding does not set that kernel's register count.
__global__ void __launch_bounds__(256, 4) eam_embed(int n_atoms, const int *__restrict__ types, EamDev E, double4 *__restrict__ pk,
                          double *__restrict__ aux, Chk ck) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_atoms) return;
    if (!MBF_OK_IDX(ck, 41, types[i], 0, ck.ns)) return;
    double acc = aux[2 * (size_t)i];
    double rb = acc > 0.0 ? acc : 0.0;
    double F, dF;
    embed64(E, E.F_f[types[i]], rb, F, dF);
    pk[i].w = dF;
    aux[2 * (size_t)i] = dF;
    aux[2 * (size_t)i + 1] = F;
}

// Force pass over the upper half of every row: each unordered pair once.
// The pair force on i is accumulated here; the one on j (its negative) is
// written to j's own slot (j -> i) = rev(i -> j), so j's gather reads its row
// contiguously.  Energy phi and the virial of the pair go to i, the lower
// index.  SlotT is float in the mixed path (a per-pair term, accumulated in
// float64 by the gather) and double in the float64 path.
template <typename T> struct SlotVec;
template <> struct SlotVec<double> { typedef double3 type; };
template <> struct SlotVec<float> { typedef float3 type; };

template <typename T, int LPA, bool ZHOU, bool ORTHO>
__global__ void __launch_bounds__(EAM_BLOCK, sizeof(T) == 4 ? MBF_EAM_MINB : 1) eam_force(SysView S, const int *__restrict__ row_off,
                                                       const int *__restrict__ upper,
                                                       const int *__restrict__ nbr,
                                                       const int *__restrict__ rev, EamDev E,
                                                       const double4 *__restrict__ pk,
                                                       const double *__restrict__ aux,
                                                       typename SlotVec<T>::type *__restrict__ slot_f,
                                                       double *__restrict__ f_local,
                                                       double *__restrict__ per_atom, Chk ck) {
    typedef typename SlotVec<T>::type V3;
    __shared__ ZTab<T> Z;
    if (ZHOU) load_ztab<T>(E, Z);
    const int sub = threadIdx.x & (LPA - 1);
    const int gpb = EAM_BLOCK / LPA;
    const double rc = E.r_cut, rc2 = rc * rc;
    for (int base = blockIdx.x * gpb; base < S.n_atoms; base += gridDim.x * gpb) {
        int i = base + threadIdx.x / LPA;
        double fx = 0, fy = 0, fz = 0, e = 0;
        int npair = 0;
        double vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
        if (i < S.n_atoms) {
            int si = S.types[i];
            double4 pi = ld_pack(pk, i);
            T Fp_i = (T)pi.w;
            CellView<ORTHO> cv;
            cv.load(S, i);
            int end = row_off[i + 1];
            int up = upper[i];
            if (!MBF_OK_IDX(ck, 21, up, row_off[i], end + 1)) up = end;
            // two-stage prefetch: slot indices two iterations ahead, the
            // neighbour's record and species one ahead, so the record load
            // never waits on the index load of the same iteration
            int s = up + sub;
            int j0 = i, r0 = 0, j1 = i, r1 = 0;
            if (s < end && MBF_OK_IDX(ck, 22, s, 0, ck.n_slots)) {
                j0 = nbr[s];
                r0 = rev[s];
            }
            if (s + LPA < end && MBF_OK_IDX(ck, 25, s + LPA, 0, ck.n_slots)) {
                j1 = nbr[s + LPA];
                r1 = rev[s + LPA];
            }
            if (!MBF_OK_IDX(ck, 23, j0, 0, ck.n_atoms)) j0 = i;
            double4 pn = ld_pack(pk, j0);
            int tn = __ldg(S.types + j0);
            for (; s < end; s += LPA) {
                double4 pj = pn;
                int sj = tn, rs = r0;
                if (!MBF_OK_IDX(ck, 24, sj, 0, ck.ns)) sj = 0;
                if (s + LPA < end) {
                    if (!MBF_OK_IDX(ck, 26, j1, 0, ck.n_atoms)) j1 = i;
                    pn = ld_pack(pk, j1);
                    tn = __ldg(S.types + j1);
                }
                r0 = r1;
                if (s + 2 * LPA < end && MBF_OK_IDX(ck, 25, s + 2 * LPA, 0, ck.n_slots)) {
                    j1 = nbr[s + 2 * LPA];
                    r1 = rev[s + 2 * LPA];
                }
                double dx, dy, dz;
                cv.mic(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z, dx, dy, dz);
                double r2 = dx * dx + dy * dy + dz * dz;
                double px = 0, py = 0, pz = 0;
                if (r2 < rc2 && r2 > 1e-24) {
                    npair += 1;
                    T r = pair_dist<T>(r2);
                    T phi, dphi, drho_j, drho_i;
                    if (ZHOU) {
                        zhou_pair_terms<T>(Z, si, sj, r, phi, dphi, drho_j, drho_i);
                    } else {
                        double rr = sqrt(r2);
                        T rj, ri;
                        feval<T>(E, E.phi_f[si * E.ns + sj], rr, phi, dphi);
                        feval<T>(E, E.rho_f[sj], rr, rj, drho_j);
                        feval<T>(E, E.rho_f[si], rr, ri, drho_i);
                    }
                    T c = dphi + Fp_i * drho_j + (T)pj.w * drho_i;
                    double sc = (double)fdiv<T>(c, r);
                    px = sc * dx;
                    py = sc * dy;
                    pz = sc * dz;
                    fx += px;
                    fy += py;
                    fz += pz;
                    e += (double)phi;
                    vxx -= px * dx;
                    vyy -= py * dy;
                    vzz -= pz * dz;
                    vxy -= px * dy;
                    vxz -= px * dz;
                    vyz -= py * dz;
                }
                V3 w;
                w.x = (T)(-px);
                w.y = (T)(-py);
                w.z = (T)(-pz);
                if (MBF_OK_IDX(ck, 27, rs, 0, ck.n_slots)) slot_f[rs] = w;
            }
        }
        fx = group_sum<LPA>(fx);
        fy = group_sum<LPA>(fy);
        fz = group_sum<LPA>(fz);
        e = group_sum<LPA>(e);
        vxx = group_sum<LPA>(vxx);
        vyy = group_sum<LPA>(vyy);
        vzz = group_sum<LPA>(vzz);
        vxy = group_sum<LPA>(vxy);
        vxz = group_sum<LPA>(vxz);
        vyz = group_sum<LPA>(vyz);
        npair = group_sum<LPA>(npair);
        if (sub == 0 && i < S.n_atoms) {
            f_local[3 * (size_t)i] = fx;
            f_local[3 * (size_t)i + 1] = fy;
            f_local[3 * (size_t)i + 2] = fz;
            double *pa = per_atom + (size_t)i * ATOM_ACC;
            pa[0] = e + aux[2 * (size_t)i + 1];
            pa[1] = vxx; pa[2] = vxy; pa[3] = vxz;
            pa[4] = vxy; pa[5] = vyy; pa[6] = vyz;
            pa[7] = vxz; pa[8] = vyz; pa[9] = vzz;
            pa[10] = (double)npair;
        }
    }
}

// F_a = (pairs above a) + the forces its lower neighbours left in a's own
// lower slots (contiguous reads), fused with the per-structure sums
// (ChunkSums): a block per chunk of the reduction plan, 8 lanes per atom;
// besides its atom's force each group adds the atom's record (entries sub
// and sub + 8 of its 8 lanes), and the block finishes the chunk's and, if
// last, the structure's sums.
template <typename V3, int NT>
__global__ void __launch_bounds__(NT) eam_gather_reduce(const int *__restrict__ row_off,
                                                              const int *__restrict__ upper,
                                                              const V3 *__restrict__ slot_f,
                                                              const double *__restrict__ f_local,
                                                              double *__restrict__ forces, ChunkSums cs, Chk ck) {
    constexpr int LPA = 8, G = NT / LPA;
    const int c = blockIdx.x;
    const int s = cs.chunk[3 * c], a0 = cs.chunk[3 * c + 1], a1 = cs.chunk[3 * c + 2];
    const int sub = threadIdx.x & (LPA - 1), grp = threadIdx.x / LPA;
    double r0 = 0.0, r1 = 0.0;
    // the next atom's row bounds are loaded one iteration ahead
    int nb = 0, nu = 0, ne = 0;
    if (a0 + grp < a1) {
        nb = row_off[a0 + grp];
        ne = row_off[a0 + grp + 1];
        nu = upper[a0 + grp];
    }
    for (int base = a0; base < a1; base += G) {  // uniform over the block
        int a = base + grp;
        const int beg = nb, rend = ne;
        int up = nu;
        if (a + G < a1) {
            nb = row_off[a + G];
            ne = row_off[a + G + 1];
            nu = upper[a + G];
        }
        double fx = 0, fy = 0, fz = 0;
        if (a < a1) {
            if (!MBF_OK_IDX(ck, 31, up, beg, rend + 1)) up = beg;
#pragma unroll 4
            for (int q = beg + sub; q < up; q += LPA) {
                if (!MBF_OK_IDX(ck, 32, q, 0, ck.n_slots)) break;
                V3 w = slot_f[q];
                fx += (double)w.x;
                fy += (double)w.y;
                fz += (double)w.z;
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

// Site terms (engine/site_terms.py:440-479): U_i = F_i(rho-bar_i) + 1/2
// sum_j phi_ij and dU_i/dv_ij = (F'_i rho'_{s_j}(r) + 1/2 phi'(r)) v / r over
// the full row, after the density and embedding passes; v for every slot.
template <typename T, int LPA, bool ZHOU, bool ORTHO>
__global__ void __launch_bounds__(EAM_BLOCK) eam_site(SysView S, const int *__restrict__ row_off,
                                                      const int *__restrict__ nbr, EamDev E,
                                                      const double4 *__restrict__ pk,
                                                      const double *__restrict__ aux, SiteOut so, Chk ck) {
    __shared__ ZTab<T> Z;
    if (ZHOU) load_ztab<T>(E, Z);
    const int sub = threadIdx.x & (LPA - 1);
    const int gpb = EAM_BLOCK / LPA;
    const double rc = E.r_cut, rc2 = rc * rc;
    for (int base = blockIdx.x * gpb; base < S.n_atoms; base += gridDim.x * gpb) {
        int i = base + threadIdx.x / LPA;
        double e = 0.0;
        if (i < S.n_atoms) {
            int si = S.types[i];
            if (!MBF_OK_IDX(ck, 51, si, 0, ck.ns)) si = 0;
            CellView<ORTHO> cv;
            cv.load(S, i);
            double4 pi = ld_pack(pk, i);
            double Fp = aux[2 * (size_t)i];
            int end = row_off[i + 1];
            if (!MBF_OK_IDX(ck, 52, end, 0, ck.n_slots + 1)) end = row_off[i];
            for (int s = row_off[i] + sub; s < end; s += LPA) {
                int j = nbr[s];
                if (!MBF_OK_IDX(ck, 53, j, 0, ck.n_atoms)) continue;
                int sj = __ldg(S.types + j);
                if (!MBF_OK_IDX(ck, 54, sj, 0, ck.ns)) sj = 0;
                double4 pj = ld_pack(pk, j);
                double dx, dy, dz;
                cv.mic(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z, dx, dy, dz);
                double r2 = dx * dx + dy * dy + dz * dz;
                size_t o = 3 * (size_t)s;
                so.vec[o] = dx;
                so.vec[o + 1] = dy;
                so.vec[o + 2] = dz;
                double c = 0.0;
                if (r2 < rc2 && r2 > 1e-24) {
                    T phi, dphi, drho_j, drho_i;
                    if (ZHOU) {
                        zhou_pair_terms<T>(Z, si, sj, pair_dist<T>(r2), phi, dphi, drho_j, drho_i);
                    } else {
                        double rr = sqrt(r2);
                        T rj;
                        feval<T>(E, E.phi_f[si * E.ns + sj], rr, phi, dphi);
                        feval<T>(E, E.rho_f[sj], rr, rj, drho_j);
                    }
                    double r = sqrt(r2);
                    e += 0.5 * (double)phi;
                    c = (Fp * (double)drho_j + 0.5 * (double)dphi) / r;
                }
                so.dudv[o] = c * dx;
                so.dudv[o + 1] = c * dy;
                so.dudv[o + 2] = c * dz;
            }
        }
        e = group_sum<LPA>(e);
        if (sub == 0 && i < S.n_atoms) so.e[i] = e + aux[2 * (size_t)i + 1];
    }
}

template <typename T, int LPA, bool ZHOU, bool ORTHO>
static int eam_launch(const SysView &S, const mbf_nlist *nl, const EamDev &E, double4 *pk, double *aux,
                      void *slot, double *f_local, double *forces, double *per_atom, Chk ck, const SiteOut &so,
                      const ChunkSums &cs, int n_chunks, cudaStream_t st) {
    typedef typename SlotVec<T>::type V3;
    int gpb = EAM_BLOCK / LPA;
    int blocks = (S.n_atoms + gpb - 1) / gpb;
    PROF_BEGIN("eam_pack", st);
    eam_pack<<<(S.n_atoms + 255) / 256, 256, 0, st>>>(S, pk);
    PROF_END("eam_pack", st);
    int g = persistent_grid(blocks, EAM_BLOCK, (const void *)eam_density<T, LPA, ZHOU, ORTHO>);
    PROF_BEGIN("eam_density", st);
    eam_density<T, LPA, ZHOU, ORTHO><<<g, EAM_BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, E, pk, aux, ck);
    PROF_END("eam_density", st);
    MBF_CHECK_LAUNCH();
    PROF_BEGIN("eam_embed", st);
    eam_embed<<<(S.n_atoms + 255) / 256, 256, 0, st>>>(S.n_atoms, S.types, E, pk, aux, ck);
    PROF_END("eam_embed", st);
    MBF_CHECK_LAUNCH();
    g = persistent_grid(blocks, EAM_BLOCK, (const void *)eam_force<T, LPA, ZHOU, ORTHO>);
    PROF_BEGIN("eam_force", st);
    eam_force<T, LPA, ZHOU, ORTHO><<<g, EAM_BLOCK, 0, st>>>(S, nl->row_off, nl->upper, nl->nbr, nl->rev, E, pk,
                                                     aux, (V3 *)slot, f_local, per_atom, ck);
    PROF_END("eam_force", st);
    MBF_CHECK_LAUNCH();
    PROF_BEGIN("eam_gather_reduce", st);
    int nt = chunk_block(S.n_atoms, n_chunks);
    if (nt == 128)
        eam_gather_reduce<V3, 128><<<n_chunks, 128, 0, st>>>(nl->row_off, nl->upper, (const V3 *)slot, f_local,
                                                              forces, cs, ck);
    else if (nt == 256)
        eam_gather_reduce<V3, 256><<<n_chunks, 256, 0, st>>>(nl->row_off, nl->upper, (const V3 *)slot, f_local,
                                                              forces, cs, ck);
    else
        eam_gather_reduce<V3, 512><<<n_chunks, 512, 0, st>>>(nl->row_off, nl->upper, (const V3 *)slot, f_local,
                                                              forces, cs, ck);
    PROF_END("eam_gather_reduce", st);
    MBF_CHECK_LAUNCH();
    if (so.e) {
        g = persistent_grid(blocks, EAM_BLOCK, (const void *)eam_site<T, LPA, ZHOU, ORTHO>);
        eam_site<T, LPA, ZHOU, ORTHO><<<g, EAM_BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, E, pk, aux, so, ck);
        MBF_CHECK_LAUNCH();
    }
    return MBF_OK;
}

template <typename T, bool ZHOU, bool ORTHO>
static int eam_dispatch_lpa(int lpa, const SysView &S, const mbf_nlist *nl, const EamDev &E, double4 *pk,
                            double *aux, void *slot, double *f_local, double *forces, double *per_atom,
                            Chk ck, const SiteOut &so, const ChunkSums &cs, int n_chunks, cudaStream_t st) {
#define MBF_EAM_LAUNCH(L) \
    eam_launch<T, L, ZHOU, ORTHO>(S, nl, E, pk, aux, slot, f_local, forces, per_atom, ck, so, cs, n_chunks, st)
    switch (lpa) {
        case 1: return MBF_EAM_LAUNCH(1);
        case 2: return MBF_EAM_LAUNCH(2);
        case 4: return MBF_EAM_LAUNCH(4);
        case 8: return MBF_EAM_LAUNCH(8);
        case 16: return MBF_EAM_LAUNCH(16);
        case 32: return MBF_EAM_LAUNCH(32);
        default: return MBF_ERR_ARGUMENT;
    }
#undef MBF_EAM_LAUNCH
}

template <typename T>
static int eam_dispatch(bool zhou, int lpa, const SysView &S, const mbf_nlist *nl, const EamDev &E,
                        double4 *pk, double *aux, void *slot, double *f_local, double *forces,
                        double *per_atom, Chk ck, const SiteOut &so, const ChunkSums &cs, int n_chunks,
                        cudaStream_t st) {
#define MBF_EAM_ARGS lpa, S, nl, E, pk, aux, slot, f_local, forces, per_atom, ck, so, cs, n_chunks, st
    if (zhou)
        return S.ortho ? eam_dispatch_lpa<T, true, true>(MBF_EAM_ARGS) : eam_dispatch_lpa<T, true, false>(MBF_EAM_ARGS);
    return S.ortho ? eam_dispatch_lpa<T, false, true>(MBF_EAM_ARGS) : eam_dispatch_lpa<T, false, false>(MBF_EAM_ARGS);
#undef MBF_EAM_ARGS
}

}  // namespace mbf

using namespace mbf;

static int eam_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
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
    SysView S = make_view(sys);
    EamDev E;
    E.ns = tab->ns; E.nf = tab->nf; E.nX = tab->nX;
    E.codes = tab->codes; E.P = tab->P; E.xo = tab->xo; E.nx = tab->nx;
    E.X = tab->X; E.C = tab->C;
    E.rho_f = tab->rho_f; E.F_f = tab->F_f; E.phi_f = tab->phi_f;
    E.r_cut = tab->r_cut;
    if (!nl->upper) return MBF_ERR_ARGUMENT;
    double *aux = ws_at<double>(workspace, L.atom_aux);
    double *per_atom = ws_at<double>(workspace, L.per_atom);
    double *partial = ws_at<double>(workspace, L.partial);
    void *slot_f = ws_at<char>(workspace, L.slot);
    Chk ck;
    ck.err = ws_at<int>(workspace, L.err);
    ck.n_atoms = sys->n_atoms;
    if (nl->n_slots < 0 || nl->n_slots > 0x7fffff00LL) return MBF_ERR_ARGUMENT;
    ck.n_slots = (int)nl->n_slots;
    ck.ns = tab->ns;
    if (cudaMemsetAsync(ck.err, 0, ERR_CLEAR_BYTES, st) != cudaSuccess) return MBF_ERR_CUDA;
    double *f_local = ws_at<double>(workspace, L.f_local);
    double4 *pk = ws_at<double4>(workspace, L.pack);
    int lpa = lanes_per_atom > 0 ? lanes_per_atom : 8;
    bool zhou = tab->zhou_fused != 0 && tab->ns <= EAM_MAXSP;
    ChunkSums cs = {plan->chunk, plan->chunk_first, per_atom, partial, energy, virial,
                    ws_at<unsigned>(workspace, L.sdone)};
    if (plan->n_chunks <= 0) return MBF_ERR_ARGUMENT;
    if (cudaMemsetAsync(cs.sdone, 0, sizeof(unsigned) * (size_t)sys->n_struct, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    if (precision == MBF_FP64)
        return eam_dispatch<double>(zhou, lpa, S, nl, E, pk, aux, slot_f, f_local, forces, per_atom, ck, so, cs,
                                    plan->n_chunks, st);
    return eam_dispatch<float>(zhou, lpa, S, nl, E, pk, aux, slot_f, f_local, forces, per_atom, ck, so, cs,
                               plan->n_chunks, st);
}

extern "C" int mbf_eam_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                            const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                            void *workspace, size_t workspace_bytes, double *forces, double *energy,
                            double *virial, void *stream) {
    SiteOut none = {nullptr, nullptr, nullptr};
    return eam_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, forces, energy,
                    virial, none, stream);
}

extern "C" int mbf_eam_eval_sites(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                                  const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                                  size_t workspace_bytes, double *forces, double *energy, double *virial,
                                  double *site_e, double *site_dudv, double *site_vec, void *stream) {
    if (!site_e || !site_dudv || !site_vec) return MBF_ERR_ARGUMENT;
    SiteOut so = {site_e, site_dudv, site_vec};
    return eam_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, forces, energy,
                    virial, so, stream);
}

// ---- the same evaluation without any allocation -----------------------------
//
// Some callers cannot allocate device memory: a host program that owns the
// whole device memory budget and hands its plug-ins only input and output
// buffers, or a time-step loop that must not synchronise the device the way
// cudaMalloc / cudaFree can.  mbf_eam_eval_static serves them: its scratch is
// this file-scope device array, reserved when the library is loaded and held
// by every GPU that loads the library until the process exits.

#define MBF_STATIC_SCRATCH_BYTES MBF_EAM_STATIC_SCRATCH_BYTES

static __device__ __align__(256) unsigned char g_eam_scratch[MBF_STATIC_SCRATCH_BYTES];

namespace mbf {

// Device address of g_eam_scratch, looked up once per device.  Host code
// must not use the array's name as a pointer: on the host it is only a
// stand-in symbol, not a device address.
static std::mutex g_scratch_mu;
static void *g_scratch_ptr[64];

static int scratch_address(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MBF_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_eam_scratch) != cudaSuccess || !p) return MBF_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return MBF_OK;
}

}  // namespace mbf

extern "C" int mbf_eam_eval_static(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                                   const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                                   double *forces, double *energy, double *virial, void *stream) {
    if (!sys || !nl || !tab || !plan || !forces || !energy || !virial) return MBF_ERR_ARGUMENT;
    if (precision != MBF_FP64 && precision != MBF_MIXED) return MBF_ERR_ARGUMENT;
    if (nl->n_atoms != sys->n_atoms || tab->ns <= 0) return MBF_ERR_ARGUMENT;
    EvalLayout L = eval_layout(sys->n_atoms, nl->n_slots, plan->n_chunks);
    if (L.total > (size_t)MBF_STATIC_SCRATCH_BYTES) return MBF_ERR_SCRATCH_LIMIT;
    void *workspace = nullptr;
    int rc = scratch_address(&workspace);
    if (rc != MBF_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (sys->n_atoms == 0) {
        if (cudaMemsetAsync(energy, 0, sizeof(double) * sys->n_struct, st) != cudaSuccess) return MBF_ERR_CUDA;
        if (cudaMemsetAsync(virial, 0, sizeof(double) * 9 * sys->n_struct, st) != cudaSuccess) return MBF_ERR_CUDA;
        return MBF_OK;
    }
    SysView S = make_view(sys);
    EamDev E;
    E.ns = tab->ns; E.nf = tab->nf; E.nX = tab->nX;
    E.codes = tab->codes; E.P = tab->P; E.xo = tab->xo; E.nx = tab->nx;
    E.X = tab->X; E.C = tab->C;
    E.rho_f = tab->rho_f; E.F_f = tab->F_f; E.phi_f = tab->phi_f;
    E.r_cut = tab->r_cut;
    if (!nl->upper) return MBF_ERR_ARGUMENT;
    double *aux = ws_at<double>(workspace, L.atom_aux);
    double *per_atom = ws_at<double>(workspace, L.per_atom);
    double *partial = ws_at<double>(workspace, L.partial);
    void *slot_f = ws_at<char>(workspace, L.slot);
    Chk ck;
    ck.err = ws_at<int>(workspace, L.err);
    ck.n_atoms = sys->n_atoms;
    if (nl->n_slots < 0 || nl->n_slots > 0x7fffff00LL) return MBF_ERR_ARGUMENT;
    ck.n_slots = (int)nl->n_slots;
    ck.ns = tab->ns;
    // the scratch keeps the previous call's contents: the error words must
    // start at zero (the reduction clears its own counters); every other
    // region is fully written before it is read
    if (cudaMemsetAsync(ck.err, 0, ERR_CLEAR_BYTES, st) != cudaSuccess) return MBF_ERR_CUDA;
    double *f_local = ws_at<double>(workspace, L.f_local);
    double4 *pk = ws_at<double4>(workspace, L.pack);
    int lpa = lanes_per_atom > 0 ? lanes_per_atom : 8;
    bool zhou = tab->zhou_fused != 0 && tab->ns <= EAM_MAXSP;
    ChunkSums cs = {plan->chunk, plan->chunk_first, per_atom, partial, energy, virial,
                    ws_at<unsigned>(workspace, L.sdone)};
    if (plan->n_chunks <= 0) return MBF_ERR_ARGUMENT;
    if (cudaMemsetAsync(cs.sdone, 0, sizeof(unsigned) * (size_t)sys->n_struct, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    if (precision == MBF_FP64)
        return eam_dispatch<double>(zhou, lpa, S, nl, E, pk, aux, slot_f, f_local, forces, per_atom, ck, SiteOut{},
                                    cs, plan->n_chunks, st);
    return eam_dispatch<float>(zhou, lpa, S, nl, E, pk, aux, slot_f, f_local, forces, per_atom, ck, SiteOut{}, cs,
                               plan->n_chunks, st);
}
