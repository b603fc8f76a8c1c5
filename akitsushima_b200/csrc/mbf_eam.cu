// Alloy EAM: energy, forces and virial of the DYNAMO / setfl alloy form over
// the two-way CSR neighbour list, in four passes, with no float atomics.
//
// Replaces engine/eam.py:174-256 and engine/_eam_kernels.py:231-307.  The
// reference visits each half pair once per phase in four serial phases
// (density, embedding, pair forces, scatter).  Here every pass is a lane
// group (or a thread) per atom over its own row:
//   eam_density   rho-bar_i = sum over i's full row of rho_{s_j}(r) (owner
//                 computes: a pair's density is evaluated from both sides,
//                 each side only the other atom's species, and nothing is
//                 scattered);
//   eam_embed     rho-bar clamped at 0, F and F' in float64 (a thread per
//                 atom), and the record {x, y, z, F'} every neighbour
//                 gathers in the force pass;
//   eam_force     each unordered pair once (the upper half of every row): its
//                 force, energy and virial go to i, the negated force to j's
//                 own slot (j -> i) = rev(i -> j);
//   eam_gather_reduce  F_j = j's upper-pair sum + the forces its lower
//                 neighbours left in its lower slots (contiguous), fused with
//                 the per-structure energy / virial sums.
// rho-bar and F(rho-bar) are float64 in both precisions.
#include <cmath>
#include <cstring>
#include <mutex>
#include <type_traits>

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
// With the cell as a launch argument (CellView<2>) the kernels need fewer
// registers: the force pass fits seven blocks per SM at 68 (74 at six,
// where it measured 126.0 against 123.2 us), the density pass twelve at 40.
#ifndef MBF_EAM_MINB_BOX
#define MBF_EAM_MINB_BOX 7
#endif
#ifndef MBF_EAM_DENS_MINB_BOX
#define MBF_EAM_DENS_MINB_BOX 12
#endif
// The same for the float32 density kernel (47 registers, no spills).
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

// Checks on every index the kernels read from the list or the species array
// before they dereference it.  A failed check substitutes an in-range index
// (or skips the store), sets the lane's flag, and the row's end records
// (site, atom) in the workspace error words 1 and 2 once; mbf_eval_status()
// returns them to the host.  They are always compiled in.  Each is one
// unsigned comparison: the entries refuse lists of more than 0x7fffff00
// slots, so every index and bound fits an int.
struct Chk {
    int *err;
    int n_atoms;
    int n_slots;
    int ns;
};

__device__ __forceinline__ int chk_idx(int v, int n, int fallback, int &flag) {
    const bool ok = (unsigned)v < (unsigned)n;
    flag |= ok ? 0 : 1;
    return ok ? v : fallback;
}

// 0 <= beg <= up <= end <= n_slots, each step one unsigned comparison.
__device__ __forceinline__ bool row_ok(int beg, int up, int end, int n_slots) {
    return (unsigned)beg <= (unsigned)up && (unsigned)up <= (unsigned)end && (unsigned)end <= (unsigned)n_slots;
}

__device__ __forceinline__ void chk_flush(const Chk &ck, int flag, int site, int atom) {
    if (flag && atomicCAS(ck.err + 1, 0, site) == 0) ck.err[2] = atom;
}

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

// ---- fused Zhou alloy path, up to EAM_MAXSP elements (shared memory) --------
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

// ---- one- and two-element Zhou path: constants as kernel arguments ---------
// For the common alloy sizes the element constants travel in the kernel's
// parameter block, so every use is an operand of the instruction itself (no
// load, no shared memory), and both elements are evaluated for every pair
// without a branch on the species.  In float32 the exponentials, reciprocals
// and the root are the PTX approximations (ex2 / rcp / rsqrt .approx, about
// 2^-22 relative); float64 keeps exp and IEEE division.

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// x clamped to [0, 1]: a saturating multiply in float32
__device__ __forceinline__ float sat01(float x) { return __saturatef(x); }
__device__ __forceinline__ double sat01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

// One element's constants (x = r / r_e).  In float32 exp(-beta (x - 1)) is
// 2^(eb (r - r_e)) with eb = -beta log2(e) / r_e: r - r_e is exact for r
// within a factor two of r_e (Sterbenz), so near the equilibrium distance,
// where the terms are largest, the argument carries only eb's own rounding
// times a small number -- no cancellation between two large constants;
// likewise alpha (ea).
template <typename T>
struct ZEl {
    T ire, re, lam, kap, beta, alpha, eb, ea, fe, fe_ire, A, B;
    T lfe;  // log2 f_e (f_e > 0): the density's prefactor moved into its exponent
};

template <typename T>
struct ZK {
    ZEl<T> el[2];
    T half_chi;       // chi / 2 of the cross pair
    T r0, iw, m30iw;  // switch: s = (r - (r_c - w)) / w; dS factor -30 / w
};

// g = exp(-expo (x - 1)) / (1 + (x - shift)^20) and h with dg/dr = -g h / r_e,
// h = expo + 20 (x - shift)^19 / (1 + (x - shift)^20) (engine/eam_zhou.py's
// decay and its derivative).
// dre = r - r_e, el = the float32 exponent factor (eb or ea).
__device__ __forceinline__ void zdec(float r, float dre, float ire, float shift, float el, float expo,
                                     float &g, float &h) {
    float u = fmaf(r, ire, -shift);
    float u2 = u * u, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8;
    float u19 = u16 * u2 * u;
    float rd = rcp_approx(fmaf(u16, u4, 1.0f));
    g = ex2_approx(el * dre) * rd;
    h = fmaf(20.0f * u19, rd, expo);
}
__device__ __forceinline__ void zdec(double r, double, double ire, double shift, double, double expo,
                                     double &g, double &h) {
    double x = r * ire, u = x - shift;
    double u2 = u * u, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8;
    double u19 = u16 * u2 * u;
    double rd = 1.0 / (1.0 + u16 * u4);
    g = exp(-expo * (x - 1.0)) * rd;
    h = expo + 20.0 * u19 * rd;
}
__device__ __forceinline__ double zval(double r, double, double ire, double shift, double, double expo) {
    double x = r * ire, u = x - shift;
    double u2 = u * u, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8;
    return exp(-expo * (x - 1.0)) / (1.0 + u16 * u4);
}

__device__ __forceinline__ void dist_ir(double r2, float &r, float &ir) {
    float q = (float)r2;
    ir = rsqrt_approx(q);
    r = q * ir;
}
__device__ __forceinline__ void dist_ir(double r2, double &r, double &ir) {
    r = sqrt(r2);
    ir = 1.0 / r;
}

// ---- evaluation policies ----------------------------------------------------
// A policy gives, for a pair inside the cutoff at squared distance r2 of
// species (si, sj):
//   dens1: the switched density rho_{s_j}(r) neighbour j puts on atom i;
//   pair: the switched pair function phi_{s_i s_j}(r) and its r-derivative,
//         the r-derivatives of the switched rho_{s_j} and rho_{s_i}, and 1 / r.
// PolGeneric reads any table (splines and every Zhou form, per call);
// PolZSmem the fused Zhou path for up to EAM_MAXSP elements (parameters in
// shared memory); PolZ2<NS> the one- or two-element Zhou path with its
// constants as kernel arguments.

template <typename T>
struct PolGeneric {
    static constexpr bool species_addresses = true;  // species index the tables
    EamDev E;
    __device__ __forceinline__ void setup(ZTab<T> &) const {}
    __device__ __forceinline__ T dens1(const ZTab<T> &, int sj, double r2) const {
        T v, dv;
        feval<T>(E, E.rho_f[sj], sqrt(r2), v, dv);
        return v;
    }
    __device__ __forceinline__ void pair(const ZTab<T> &, int si, int sj, double r2, T &phi, T &dphi, T &drj,
                                         T &dri, T &ir) const {
        double rr = sqrt(r2);
        T v;
        feval<T>(E, E.phi_f[si * E.ns + sj], rr, phi, dphi);
        feval<T>(E, E.rho_f[sj], rr, v, drj);
        dri = drj;
        if (si != sj) feval<T>(E, E.rho_f[si], rr, v, dri);
        ir = (T)(1.0 / rr);
    }
};

template <typename T>
__device__ __forceinline__ T pair_dist(double r2);
template <> __device__ __forceinline__ double pair_dist<double>(double r2) { return sqrt(r2); }
template <> __device__ __forceinline__ float pair_dist<float>(double r2) { return sqrtf((float)r2); }

template <typename T>
struct PolZSmem {
    static constexpr bool species_addresses = true;  // species index the tables
    EamDev E;
    __device__ __forceinline__ void setup(ZTab<T> &Z) const { load_ztab<T>(E, Z); }
    __device__ __forceinline__ T dens1(const ZTab<T> &Z, int sj, double r2) const {
        T r = pair_dist<T>(r2);
        T S, dS;
        zswitch_fast<T>(r, Z, S, dS);
        return zdens_only<T>(Z.sp[sj], r) * S;
    }
    __device__ __forceinline__ void pair(const ZTab<T> &Z, int si, int sj, double r2, T &phi, T &dphi, T &drj,
                                         T &dri, T &ir) const {
        T r = pair_dist<T>(r2);
        zhou_pair_terms<T>(Z, si, sj, r, phi, dphi, drj, dri);
        ir = fdiv<T>(T(1), r);
    }
};

// The float32 switched density rho_{s_j}(r) of the one- and two-element
// paths: S(r) 2^(eb (r - r_e) + log2 f_e) / (1 + (r / r_e - lambda)^20),
// the prefactor in the exponent (one multiply fewer per slot), r from one
// sqrt.approx (no 1 / r needed here), the switch's clamp a saturation, its
// polynomial 1 - s^3 (10 - 15 s + 6 s^2) in Horner form.
template <int NS>
__device__ __forceinline__ float zdens_f32(const ZK<float> &K, int sj, double r2) {
    const float r = sqrt_approx((float)r2);
    const ZEl<float> &a = K.el[0], &b = K.el[1];
    const bool one = NS == 1 || sj == 0;
    const float re = one ? a.re : b.re, ire = one ? a.ire : b.ire, lam = one ? a.lam : b.lam;
    const float eb = one ? a.eb : b.eb, lfe = one ? a.lfe : b.lfe;
    const float s = sat01((r - K.r0) * K.iw), s2 = s * s;
    const float S = fmaf(-s2 * s, fmaf(6.f, s2, fmaf(-15.f, s, 10.f)), 1.f);
    const float u = fmaf(r, ire, -lam);
    const float u2 = u * u, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8;
    return S * ex2_approx(fmaf(eb, r - re, lfe)) * rcp_approx(fmaf(u16, u4, 1.f));
}

template <typename T, int NS>
struct PolZ2 {
    static constexpr bool species_addresses = false;  // species only compared, never an index
    ZK<T> K;
    __device__ __forceinline__ void setup(ZTab<T> &) const {}

    __device__ __forceinline__ T sw_val(T r) const {
        const T s = sat01((r - K.r0) * K.iw);
        return T(1) - s * s * s * (T(10) - T(15) * s + T(6) * s * s);
    }
    __device__ __forceinline__ void sw(T r, T &S, T &dS) const {
        const T s = sat01((r - K.r0) * K.iw);
        T s2 = s * s, om = T(1) - s;
        S = T(1) - s2 * s * (T(10) - T(15) * s + T(6) * s2);
        dS = K.m30iw * s2 * om * om;
    }
    // f = f_e gB, phi_aa = A gA - B gB and their r-derivatives, unswitched.
    __device__ __forceinline__ void element(const ZEl<T> &p, T r, T &f, T &df, T &ph, T &dph) const {
        T gB, hB, gA, hA;
        const T dre = r - p.re;
        zdec(r, dre, p.ire, p.lam, p.eb, p.beta, gB, hB);
        zdec(r, dre, p.ire, p.kap, p.ea, p.alpha, gA, hA);
        f = p.fe * gB;
        df = -p.fe_ire * gB * hB;
        T a = p.A * gA, b = p.B * gB;
        ph = a - b;
        dph = -p.ire * (a * hA - b * hB);
    }
    // one element's switched density, its constants selected by species
    __device__ __forceinline__ T dens1(const ZTab<T> &, int sj, double r2) const {
        if constexpr (std::is_same<T, float>::value) {
            return zdens_f32<NS>(K, sj, r2);
        } else {
            T r, ir;
            dist_ir(r2, r, ir);
            const ZEl<T> &a = K.el[0], &b = K.el[1];
            const bool one = NS == 1 || sj == 0;
            const T re = one ? a.re : b.re, ire = one ? a.ire : b.ire, lam = one ? a.lam : b.lam;
            const T eb = one ? a.eb : b.eb, beta = one ? a.beta : b.beta, fe = one ? a.fe : b.fe;
            return fe * sw_val(r) * zval(r, r - re, ire, lam, eb, beta);
        }
    }
    __device__ __forceinline__ void pair(const ZTab<T> &, int si, int sj, double r2, T &phi, T &dphi, T &drj,
                                         T &dri, T &ir) const {
        T r;
        dist_ir(r2, r, ir);
        T S, dS;
        sw(r, S, dS);
        T f0, df0, p0, dp0;
        element(K.el[0], r, f0, df0, p0, dp0);
        if (NS == 1) {
            phi = p0 * S;
            dphi = dp0 * S + p0 * dS;
            drj = dri = df0 * S + f0 * dS;
            return;
        }
        T f1, df1, p1, dp1;
        element(K.el[1], r, f1, df1, p1, dp1);
        // cross pair phi_01 = chi / 2 (q phi_00 + phi_11 / q), q = f_1 / f_0,
        // from the unswitched functions (engine/eam_zhou.py:128-207)
        T inv = fdiv<T>(T(1), f0 * f1);
        T q = f1 * f1 * inv, rq = f0 * f0 * inv, rf0 = f1 * inv;
        T dq = (df1 - q * df0) * rf0;
        T v = K.half_chi * (q * p0 + p1 * rq);
        T dv = K.half_chi * (dq * p0 + q * dp0 + (dp1 - p1 * dq * rq) * rq);
        const bool cross = si != sj;
        T pv = cross ? v : (si == 0 ? p0 : p1);
        T pdv = cross ? dv : (si == 0 ? dp0 : dp1);
        phi = pv * S;
        dphi = pdv * S + pv * dS;
        T d0 = df0 * S + f0 * dS, d1 = df1 * S + f1 * dS;
        drj = sj == 0 ? d0 : d1;
        dri = si == 0 ? d0 : d1;
    }
};

// ---- the two-element float32 path on packed pairs ---------------------------
// Blackwell's paired float32 instructions (add / mul / fma .f32x2) run one
// operation on two values at once.  The two elements' decays are the same
// instruction sequence with different constants, so the pair evaluation
// packs element 0 and element 1 into the two halves of a 64-bit register:
// the polynomial and product steps take half the instructions; the
// exponentials and reciprocals stay per element (no paired form).

typedef unsigned long long f2x;
__device__ __forceinline__ f2x pk2(float lo, float hi) {
    f2x r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void up2(f2x v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) {
    f2x d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2x mul2(f2x a, f2x b) {
    f2x d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2x add2(f2x a, f2x b) {
    f2x d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Packed constants (element 0 low, element 1 high), built on the host.
struct ZK2x {
    f2x ire, nre, nlam, nkap, eb, ea, beta, alpha, fe, nfe_ire, A, nB, nire, one, twenty;
};

static inline f2x pack_host(float lo, float hi) {
    unsigned int a, b;
    memcpy(&a, &lo, 4);
    memcpy(&b, &hi, 4);
    return (f2x)a | ((f2x)b << 32);
}

// g and h of both elements' decays with the same exponent / shift pairs.
__device__ __forceinline__ void zdec2(f2x r2, f2x dre, f2x ire, f2x nshift, f2x el, f2x expo, f2x twenty, f2x one,
                                      f2x &g, f2x &h) {
    const f2x u = fma2(r2, ire, nshift);
    const f2x u2 = mul2(u, u), u4 = mul2(u2, u2), u8 = mul2(u4, u4), u16 = mul2(u8, u8);
    const f2x u19 = mul2(mul2(u16, u2), u);
    const f2x d = fma2(u16, u4, one);
    const f2x arg = mul2(el, dre);
    float d0, d1, a0, a1;
    up2(d, d0, d1);
    up2(arg, a0, a1);
    const f2x rd = pk2(rcp_approx(d0), rcp_approx(d1));
    g = mul2(pk2(ex2_approx(a0), ex2_approx(a1)), rd);
    h = fma2(mul2(twenty, u19), rd, expo);
}

struct PolZ2x {
    static constexpr bool species_addresses = false;  // species only compared, never an index
    ZK<float> K;
    ZK2x X;
    __device__ __forceinline__ void setup(ZTab<float> &) const {}
    __device__ __forceinline__ float dens1(const ZTab<float> &, int sj, double r2) const {
        return zdens_f32<2>(K, sj, r2);
    }
    __device__ __forceinline__ void pair(const ZTab<float> &, int si, int sj, double r2, float &phi, float &dphi,
                                         float &drj, float &dri, float &ir) const {
        float r;
        dist_ir(r2, r, ir);
        const float s = sat01((r - K.r0) * K.iw);
        const float s2 = s * s, om = 1.f - s;
        const float S = 1.f - s2 * s * (10.f - 15.f * s + 6.f * s2);
        const float dS = K.m30iw * s2 * om * om;
        const f2x rr = pk2(r, r);
        const f2x dre = add2(rr, X.nre);
        f2x gB, hB, gA, hA;
        zdec2(rr, dre, X.ire, X.nlam, X.eb, X.beta, X.twenty, X.one, gB, hB);
        zdec2(rr, dre, X.ire, X.nkap, X.ea, X.alpha, X.twenty, X.one, gA, hA);
        const f2x f = mul2(X.fe, gB);
        const f2x df = mul2(mul2(X.nfe_ire, gB), hB);
        const f2x av = mul2(X.A, gA), nb = mul2(X.nB, gB);
        const f2x ph = add2(av, nb);
        const f2x dph = mul2(X.nire, fma2(nb, hB, mul2(av, hA)));
        float f0, f1, df0, df1, p0, p1, dp0, dp1;
        up2(f, f0, f1);
        up2(df, df0, df1);
        up2(ph, p0, p1);
        up2(dph, dp0, dp1);
        // cross pair phi_01 = chi / 2 (q phi_00 + phi_11 / q), q = f_1 / f_0,
        // from the unswitched functions (engine/eam_zhou.py:128-207)
        const float inv = rcp_approx(f0 * f1);
        const float q = f1 * f1 * inv, rq = f0 * f0 * inv, rf0 = f1 * inv;
        const float dq = (df1 - q * df0) * rf0;
        const float v = K.half_chi * (q * p0 + p1 * rq);
        const float dv = K.half_chi * (dq * p0 + q * dp0 + (dp1 - p1 * dq * rq) * rq);
        const bool cross = si != sj;
        const float pv = cross ? v : (si == 0 ? p0 : p1);
        const float pdv = cross ? dv : (si == 0 ? dp0 : dp1);
        phi = pv * S;
        dphi = pdv * S + pv * dS;
        const float d0 = df0 * S + f0 * dS, d1 = df1 * S + f1 * dS;
        drj = sj == 0 ? d0 : d1;
        dri = si == 0 ? d0 : d1;
    }
};

static bool make_zk2x(const ZK<float> &K, ZK2x &X) {
    const ZEl<float> &a = K.el[0], &b = K.el[1];
    X.ire = pack_host(a.ire, b.ire);
    X.nre = pack_host(-a.re, -b.re);
    X.nlam = pack_host(-a.lam, -b.lam);
    X.nkap = pack_host(-a.kap, -b.kap);
    X.eb = pack_host(a.eb, b.eb);
    X.ea = pack_host(a.ea, b.ea);
    X.beta = pack_host(a.beta, b.beta);
    X.alpha = pack_host(a.alpha, b.alpha);
    X.fe = pack_host(a.fe, b.fe);
    X.nfe_ire = pack_host(-a.fe_ire, -b.fe_ire);
    X.A = pack_host(a.A, b.A);
    X.nB = pack_host(-a.B, -b.B);
    X.nire = pack_host(-a.ire, -b.ire);
    X.one = pack_host(1.0f, 1.0f);
    X.twenty = pack_host(20.0f, 20.0f);
    return true;
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

// The cell of one atom as the force kernels need it.  CM 0: any cell (the
// 3x3 pair from global memory); CM 1: a diagonal cell, six scalars
// (lengths and inverse lengths) in registers; CM 2: one diagonal cell whose
// six scalars came with the launch (SysView::box, read from the parameter
// space where they are used: twelve registers fewer, so more resident warps).
template <int CM>
struct CellView {
    const double *c;
    double L0, L1, L2, i0, i1, i2;
    const SysView *S_;
    __device__ __forceinline__ void load(const SysView &S, int atom) {
        if (CM == 2) {
            S_ = &S;
            return;
        }
        c = cell_of(S, atom);
        if (CM == 1) {
            L0 = c[0]; L1 = c[4]; L2 = c[8];
            i0 = c[9]; i1 = c[13]; i2 = c[17];
        }
    }
    __device__ __forceinline__ void mic(double rx, double ry, double rz, double &dx, double &dy,
                                        double &dz) const {
        if (CM == 2) {
            dx = rx - S_->box[0] * rint_shift(rx * S_->box[3]);
            dy = ry - S_->box[1] * rint_shift(ry * S_->box[4]);
            dz = rz - S_->box[2] * rint_shift(rz * S_->box[5]);
        } else if (CM == 1) {
            dx = rx - L0 * rint_shift(rx * i0);
            dy = ry - L1 * rint_shift(ry * i1);
            dz = rz - L2 * rint_shift(rz * i2);
        } else {
            mic_fast(c, rx, ry, rz, dx, dy, dz);
        }
    }
};

// ---- kernels --------------------------------------------------------------

// The gather reads each pair force once: a streaming load (evict-first),
// so the forces do not displace the per-atom records from the caches
// (60 against 66.6 us at 256k).
__device__ __forceinline__ float4 ld_slot(const float4 *p) { return __ldcs(p); }
__device__ __forceinline__ double3 ld_slot(const double3 *p) { return *p; }

__device__ __forceinline__ double4 ld_pack(const double4 *__restrict__ pk, int j) {
    const double2 *p = reinterpret_cast<const double2 *>(pk + j);
    double2 a = __ldg(p), b = __ldg(p + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ double3 ld_pos(const double *__restrict__ pos, int j) {
    const double *p = pos + 3 * (size_t)j;
    return make_double3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// rho-bar_i = sum over i's full row of the switched rho_{s_j}(r) (owner
// computes, engine/_eam_kernels.py:241-273: the density at an atom comes
// from its neighbours' species functions), accumulated in float64 into
// aux[2 i].  Slot indices are loaded two iterations ahead, the neighbour's
// position and species one ahead.
template <typename T, int LPA, class Pol, int CM>
__global__ void __launch_bounds__(EAM_BLOCK, sizeof(T) == 4 ? (CM == 2 ? MBF_EAM_DENS_MINB_BOX : MBF_EAM_DENS_MINB) : 1)
    eam_density(SysView S, const int *__restrict__ row_off, const int *__restrict__ nbr, Pol P, double rc2,
                double *__restrict__ aux, Chk ck) {
    __shared__ ZTab<T> Z;
    P.setup(Z);
    const int sub = threadIdx.x & (LPA - 1);
    const int gpb = EAM_BLOCK / LPA;
    for (int base = blockIdx.x * gpb; base < S.n_atoms; base += gridDim.x * gpb) {
        const int i = base + threadIdx.x / LPA;
        double acc = 0.0;
        if (i < S.n_atoms) {
            int flag = 0;
            int beg = row_off[i], end = row_off[i + 1];
            if (!row_ok(beg, beg, end, ck.n_slots)) {
                flag = 1;
                beg = end = 0;
            }
            CellView<CM> cv;
            cv.load(S, i);
            const double3 pi = ld_pos(S.pos, i);
            int s = beg + sub;
            int j0 = i, j1 = i;
            if (s < end) j0 = nbr[s];
            if (s + LPA < end) j1 = nbr[s + LPA];
            j0 = chk_idx(j0, ck.n_atoms, i, flag);
            double3 pn = ld_pos(S.pos, j0);
            int tn = __ldg(S.types + j0);
            for (; s < end; s += LPA) {
                const double3 pj = pn;
                // a species that indexes no memory needs no check here: the
                // embedding pass checks every atom's species
                const int sj = Pol::species_addresses ? chk_idx(tn, ck.ns, 0, flag) : tn;
                if (s + LPA < end) {
                    j1 = chk_idx(j1, ck.n_atoms, i, flag);
                    pn = ld_pos(S.pos, j1);
                    tn = __ldg(S.types + j1);
                }
                if (s + 2 * LPA < end) j1 = nbr[s + 2 * LPA];
                double dx, dy, dz;
                cv.mic(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z, dx, dy, dz);
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < rc2 && r2 > 1e-24) acc += (double)P.dens1(Z, sj, r2);
            }
            chk_flush(ck, flag, 11, i);
        }
        acc = group_sum<LPA>(acc);
        if (sub == 0 && i < S.n_atoms) aux[2 * (size_t)i] = acc;
    }
}

// F(rho-bar) and F'(rho-bar) in float64, rho-bar clamped at 0
// (engine/_eam_kernels.py:268-274), and the record {x, y, z, F'} every
// neighbour reads in the force pass (one 32-byte sector per gather); a
// thread per atom, kept out of the density loop so the float64 pow / log of
// the embedding does not set that kernel's register count.
__global__ void __launch_bounds__(256, 4) eam_embed(SysView S, EamDev E, double4 *__restrict__ pk,
                                                    double *__restrict__ aux, Chk ck) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= S.n_atoms) return;
    int flag = 0;
    const int t = chk_idx(__ldg(S.types + a), ck.ns, 0, flag);
    double rb = aux[2 * (size_t)a];
    rb = rb > 0.0 ? rb : 0.0;
    double F, dF;
    embed64(E, E.F_f[t], rb, F, dF);
    const double3 p = ld_pos(S.pos, a);
    pk[a] = make_double4(p.x, p.y, p.z, dF);
    aux[2 * (size_t)a] = dF;
    aux[2 * (size_t)a + 1] = F;
    chk_flush(ck, flag, 41, a);
}

// The pair force one atom leaves in its partner's reverse slot: float4 in
// the mixed path (one aligned 16-byte store and load), double3 in float64.
template <typename T> struct SlotVec;
template <> struct SlotVec<double> {
    typedef double3 type;
    static __device__ __forceinline__ type make(double x, double y, double z) { return make_double3(x, y, z); }
};
template <> struct SlotVec<float> {
    typedef float4 type;
    static __device__ __forceinline__ type make(float x, float y, float z) { return make_float4(x, y, z, 0.0f); }
};

// Force pass over the upper half of every row: each unordered pair once.
// c = phi' + F'_i rho'_{s_j} + F'_j rho'_{s_i}; the pair force (c / r) d on i
// (d = r_j - r_i, minimum image), the pair energy and the virial -f (x) d go
// to i, the lower index; -f goes to j's own slot (j -> i) = rev(i -> j), so
// j's gather reads its row contiguously (0 beyond the cutoff).  T is float
// in the mixed path (the pair terms, and each lane's sums over its quarter
// of the row, at most about 20 terms; float64 across lanes and in the
// gather) and double in the float64 path.
template <typename T, int LPA, class Pol, int CM>
__global__ void __launch_bounds__(EAM_BLOCK, sizeof(T) == 4 ? (CM == 2 ? MBF_EAM_MINB_BOX : MBF_EAM_MINB) : 1)
    eam_force(SysView S, const int *__restrict__ row_off, const int *__restrict__ upper,
              const int *__restrict__ nbr, const int *__restrict__ rev, Pol P, double rc2,
              const double4 *__restrict__ pk, const double *__restrict__ aux,
              typename SlotVec<T>::type *__restrict__ slot_f, double *__restrict__ f_local,
              double *__restrict__ per_atom, Chk ck) {
    __shared__ ZTab<T> Z;
    P.setup(Z);
    const int sub = threadIdx.x & (LPA - 1);
    const int gpb = EAM_BLOCK / LPA;
    for (int base = blockIdx.x * gpb; base < S.n_atoms; base += gridDim.x * gpb) {
        const int i = base + threadIdx.x / LPA;
        // this lane's sums over its pairs (T: at most a row's upper half / LPA
        // terms in float32 in the mixed path), float64 from the lane sums on
        T afx = 0, afy = 0, afz = 0, ae = 0;
        T axx = 0, ayy = 0, azz = 0, axy = 0, axz = 0, ayz = 0;
        int npair = 0;
        if (i < S.n_atoms) {
            int flag = 0;
            int up = upper[i], end = row_off[i + 1];
            if (!row_ok(row_off[i], up, end, ck.n_slots)) {
                flag = 1;
                up = end = 0;
            }
            const int si = chk_idx(__ldg(S.types + i), ck.ns, 0, flag);
            const double4 pi = ld_pack(pk, i);
            const T Fp_i = (T)pi.w;
            CellView<CM> cv;
            cv.load(S, i);
            int s = up + sub;
            int j0 = i, v0 = 0, j1 = i, v1 = 0;
            if (s < end) {
                j0 = nbr[s];
                v0 = rev[s];
            }
            if (s + LPA < end) {
                j1 = nbr[s + LPA];
                v1 = rev[s + LPA];
            }
            j0 = chk_idx(j0, ck.n_atoms, i, flag);
            double4 pn = ld_pack(pk, j0);
            int tn = __ldg(S.types + j0);
            for (; s < end; s += LPA) {
                const double4 pj = pn;
                // a species that indexes no memory needs no check here: the
                // embedding pass checks every atom's species
                const int sj = Pol::species_addresses ? chk_idx(tn, ck.ns, 0, flag) : tn;
                const int rs = v0;
                if (s + LPA < end) {
                    j1 = chk_idx(j1, ck.n_atoms, i, flag);
                    pn = ld_pack(pk, j1);
                    tn = __ldg(S.types + j1);
                }
                v0 = v1;
                if (s + 2 * LPA < end) {
                    j1 = nbr[s + 2 * LPA];
                    v1 = rev[s + 2 * LPA];
                }
                double dx, dy, dz;
                cv.mic(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z, dx, dy, dz);
                const double r2 = dx * dx + dy * dy + dz * dz;
                T qx = 0, qy = 0, qz = 0;  // the pair force on j
                if (r2 < rc2 && r2 > 1e-24) {
                    npair += 1;
                    T phi, dphi, drj, dri, ir;
                    P.pair(Z, si, sj, r2, phi, dphi, drj, dri, ir);
                    const T c = dphi + Fp_i * drj + (T)pj.w * dri;
                    const T sc = c * ir;
                    const T ex = (T)dx, ey = (T)dy, ez = (T)dz;
                    const T px = sc * ex, py = sc * ey, pz = sc * ez;
                    afx += px;
                    afy += py;
                    afz += pz;
                    ae += phi;
                    axx -= px * ex;
                    ayy -= py * ey;
                    azz -= pz * ez;
                    axy -= px * ey;
                    axz -= px * ez;
                    ayz -= py * ez;
                    qx = -px;
                    qy = -py;
                    qz = -pz;
                }
                if ((unsigned)rs < (unsigned)ck.n_slots) slot_f[rs] = SlotVec<T>::make(qx, qy, qz);
                else flag = 1;
            }
            chk_flush(ck, flag, 21, i);
        }
        double fx = afx, fy = afy, fz = afz, e = ae;
        double vxx = axx, vyy = ayy, vzz = azz, vxy = axy, vxz = axz, vyz = ayz;
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
// last, the structure's sums.  The kernel waits on memory, so every load of
// an atom is issued before any is used: its first GATHER_UNROLL x 8 lower
// slots (an fcc row's lower half is about 40), its record and its
// upper-pair force, with the next atom's row bounds one iteration ahead.
constexpr int GATHER_UNROLL = 5;

template <typename V3, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) eam_gather_reduce(int n_slots, const int *__restrict__ row_off,
                                                        const int *__restrict__ upper, const V3 *__restrict__ slot_f,
                                                        const double *__restrict__ f_local,
                                                        double *__restrict__ forces, ChunkSums cs, Chk ck) {
    constexpr int LPA = 8, G = NT / LPA;
    const int c = blockIdx.x;
    const int s = cs.chunk[3 * c], a0 = cs.chunk[3 * c + 1], a1 = cs.chunk[3 * c + 2];
    const int sub = threadIdx.x & (LPA - 1), grp = threadIdx.x / LPA;
    double r0 = 0.0, r1 = 0.0;
    int nb = 0, nu = 0, ne = 0;
    if (a0 + grp < a1) {
        nb = row_off[a0 + grp];
        ne = row_off[a0 + grp + 1];
        nu = upper[a0 + grp];
    }
    for (int base = a0; base < a1; base += G) {  // uniform over the block
        const int a = base + grp;
        int beg = nb, up = nu;
        const int rend = ne;
        if (a + G < a1) {
            nb = row_off[a + G];
            ne = row_off[a + G + 1];
            nu = upper[a + G];
        }
        double fx = 0, fy = 0, fz = 0, fl = 0.0;
        if (a < a1) {
            if (!row_ok(beg, up, rend, n_slots)) {
                chk_flush(ck, 1, 31, a);
                beg = up = 0;
            }
            const double *rec = cs.per_atom + (size_t)a * ATOM_ACC;
            const double ra = rec[sub];
            const double rb = sub < ATOM_ACC - LPA ? rec[LPA + sub] : 0.0;
            if (sub < 3) fl = f_local[3 * (size_t)a + sub];
            V3 w[GATHER_UNROLL];
#pragma unroll
            for (int k = 0; k < GATHER_UNROLL; ++k) {
                const int q = beg + sub + k * LPA;
                if (q < up) w[k] = ld_slot(slot_f + q);
            }
#pragma unroll
            for (int k = 0; k < GATHER_UNROLL; ++k) {
                if (beg + sub + k * LPA < up) {
                    fx += (double)w[k].x;
                    fy += (double)w[k].y;
                    fz += (double)w[k].z;
                }
            }
            for (int q = beg + sub + GATHER_UNROLL * LPA; q < up; q += LPA) {
                const V3 v = ld_slot(slot_f + q);
                fx += (double)v.x;
                fy += (double)v.y;
                fz += (double)v.z;
            }
            r0 += ra;
            r1 += rb;
        }
        fx = group_sum<LPA>(fx);
        fy = group_sum<LPA>(fy);
        fz = group_sum<LPA>(fz);
        // lane k (k < 3) of the group holds component k of the upper-pair sum
        const double gx = __shfl_sync(MBF_FULL, fl, 0, LPA);
        const double gy = __shfl_sync(MBF_FULL, fl, 1, LPA);
        const double gz = __shfl_sync(MBF_FULL, fl, 2, LPA);
        if (sub == 0 && a < a1) {
            forces[3 * (size_t)a] = gx + fx;
            forces[3 * (size_t)a + 1] = gy + fy;
            forces[3 * (size_t)a + 2] = gz + fz;
        }
    }
    chunk_sums_finish<NT>(cs, c, s, r0, r1);
}

// Site terms (engine/site_terms.py:440-479): U_i = F_i(rho-bar_i) + 1/2
// sum_j phi_ij and dU_i/dv_ij = (F'_i rho'_{s_j}(r) + 1/2 phi'(r)) v / r over
// the full row, after the density and embedding passes; v for every slot.
template <typename T, class Pol, bool ORTHO>
__global__ void __launch_bounds__(EAM_BLOCK) eam_site(SysView S, const int *__restrict__ row_off,
                                                      const int *__restrict__ nbr, Pol P, double rc2,
                                                      const double4 *__restrict__ pk,
                                                      const double *__restrict__ aux, SiteOut so, Chk ck) {
    constexpr int LPA = 8;
    __shared__ ZTab<T> Z;
    P.setup(Z);
    const int sub = threadIdx.x & (LPA - 1);
    const int gpb = EAM_BLOCK / LPA;
    for (int base = blockIdx.x * gpb; base < S.n_atoms; base += gridDim.x * gpb) {
        const int i = base + threadIdx.x / LPA;
        double e = 0.0;
        if (i < S.n_atoms) {
            int flag = 0;
            int beg = row_off[i], end = row_off[i + 1];
            if (!row_ok(beg, beg, end, ck.n_slots)) {
                flag = 1;
                beg = end = 0;
            }
            const int si = chk_idx(__ldg(S.types + i), ck.ns, 0, flag);
            CellView<ORTHO ? 1 : 0> cv;
            cv.load(S, i);
            const double4 pi = ld_pack(pk, i);
            const double Fp = aux[2 * (size_t)i];
            for (int s = beg + sub; s < end; s += LPA) {
                const int j = chk_idx(nbr[s], ck.n_atoms, i, flag);
                const int sj = chk_idx(__ldg(S.types + j), ck.ns, 0, flag);
                const double4 pj = ld_pack(pk, j);
                double dx, dy, dz;
                cv.mic(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z, dx, dy, dz);
                const double r2 = dx * dx + dy * dy + dz * dz;
                const size_t o = 3 * (size_t)s;
                so.vec[o] = dx;
                so.vec[o + 1] = dy;
                so.vec[o + 2] = dz;
                double c = 0.0;
                if (r2 < rc2 && r2 > 1e-24) {
                    T phi, dphi, drj, dri, ir;
                    P.pair(Z, si, sj, r2, phi, dphi, drj, dri, ir);
                    e += 0.5 * (double)phi;
                    c = (Fp * (double)drj + 0.5 * (double)dphi) / sqrt(r2);
                }
                so.dudv[o] = c * dx;
                so.dudv[o + 1] = c * dy;
                so.dudv[o + 2] = c * dz;
            }
            chk_flush(ck, flag, 51, i);
        }
        e = group_sum<LPA>(e);
        if (sub == 0 && i < S.n_atoms) so.e[i] = e + aux[2 * (size_t)i + 1];
    }
}

// ---- host side ----------------------------------------------------------------

struct EamBufs {
    double4 *pk;
    double *aux;
    void *slot;  // per-slot pair forces (SlotVec<T>)
    double *f_local;
    double *forces;
    double *per_atom;
};

// Phases of an evaluation: the density and embedding passes (F'(rho-bar)
// of every atom), then the force pass and the gather.  A spatially split
// structure runs them apart, with the halo atoms' F' exchanged in between.
enum { PH_EMBED = 1, PH_FORCE = 2, PH_ALL = 3 };



// The density pass walks full rows (twice the force pass's upper halves);
// it takes 4 lanes per atom, or the force pass's lanes when that is more.
template <typename T, int LPA, class Pol, int CM>
static int eam_launch(const SysView &S, const mbf_nlist *nl, const Pol &P, const EamDev &E, double rc2,
                      const EamBufs &B, Chk ck, const SiteOut &so, const ChunkSums &cs, int n_chunks,
                      int phases, cudaStream_t st) {
    typedef typename SlotVec<T>::type V3;
    constexpr int DLPA = LPA >= 4 ? LPA : 4;
    V3 *slot = static_cast<V3 *>(B.slot);
    int g = 0;
    if (phases & PH_EMBED) {
        const int dgpb = EAM_BLOCK / DLPA;
        g = persistent_grid((S.n_atoms + dgpb - 1) / dgpb, EAM_BLOCK, (const void *)eam_density<T, DLPA, Pol, CM>);
        PROF_BEGIN("eam_density", st);
        eam_density<T, DLPA, Pol, CM><<<g, EAM_BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, P, rc2, B.aux, ck);
        PROF_END("eam_density", st);
        MBF_CHECK_LAUNCH();
        PROF_BEGIN("eam_embed", st);
        eam_embed<<<(S.n_atoms + 255) / 256, 256, 0, st>>>(S, E, B.pk, B.aux, ck);
        PROF_END("eam_embed", st);
        MBF_CHECK_LAUNCH();
    }
    if (!(phases & PH_FORCE)) return MBF_OK;
    const int gpb = EAM_BLOCK / LPA;
    // one block per step of EAM_BLOCK / LPA atoms, not a persistent grid:
    // upper halves differ in length, and blocks taken up as others finish
    // leave a shorter tail than a fixed share per resident block (126.6
    // against 133.7 us at 256k; the density pass, whose full rows are
    // alike, keeps its persistent grid)
    g = (S.n_atoms + gpb - 1) / gpb;
    PROF_BEGIN("eam_force", st);
    eam_force<T, LPA, Pol, CM><<<g, EAM_BLOCK, 0, st>>>(S, nl->row_off, nl->upper, nl->nbr, nl->rev, P, rc2,
                                                           B.pk, B.aux, slot, B.f_local, B.per_atom, ck);
    PROF_END("eam_force", st);
    MBF_CHECK_LAUNCH();
    PROF_BEGIN("eam_gather_reduce", st);
    const int nt = chunk_block(S.n_atoms, n_chunks);
    if (nt == 128)
        eam_gather_reduce<V3, 128><<<n_chunks, 128, 0, st>>>(ck.n_slots, nl->row_off, nl->upper, slot, B.f_local,
                                                             B.forces, cs, ck);
    else if (nt == 256)
        eam_gather_reduce<V3, 256><<<n_chunks, 256, 0, st>>>(ck.n_slots, nl->row_off, nl->upper, slot, B.f_local,
                                                             B.forces, cs, ck);
    else
        eam_gather_reduce<V3, 512><<<n_chunks, 512, 0, st>>>(ck.n_slots, nl->row_off, nl->upper, slot, B.f_local,
                                                             B.forces, cs, ck);
    PROF_END("eam_gather_reduce", st);
    MBF_CHECK_LAUNCH();
    if (so.e) {
        g = persistent_grid((S.n_atoms + 15) / 16, EAM_BLOCK, (const void *)eam_site<T, Pol, CM != 0>);
        eam_site<T, Pol, CM != 0><<<g, EAM_BLOCK, 0, st>>>(S, nl->row_off, nl->nbr, P, rc2, B.pk, B.aux, so, ck);
        MBF_CHECK_LAUNCH();
    }
    return MBF_OK;
}

template <typename T, class Pol, int CM>
static int eam_dispatch_lpa(int lpa, const SysView &S, const mbf_nlist *nl, const Pol &P, const EamDev &E,
                            double rc2, const EamBufs &B, Chk ck, const SiteOut &so, const ChunkSums &cs,
                            int n_chunks, int phases, cudaStream_t st) {
#define MBF_EAM_LAUNCH(L) eam_launch<T, L, Pol, CM>(S, nl, P, E, rc2, B, ck, so, cs, n_chunks, phases, st)
    switch (lpa) {
        case 1: return MBF_EAM_LAUNCH(1);
        case 2: return MBF_EAM_LAUNCH(2);
        case 4: return MBF_EAM_LAUNCH(4);
        case 8: return MBF_EAM_LAUNCH(8);
        default: return MBF_ERR_ARGUMENT;
    }
#undef MBF_EAM_LAUNCH
}

template <typename T, class Pol>
static int eam_dispatch(const Pol &P, int lpa, const SysView &S, const mbf_nlist *nl, const EamDev &E, double rc2,
                        const EamBufs &B, Chk ck, const SiteOut &so, const ChunkSums &cs, int n_chunks,
                        int phases, cudaStream_t st) {
    // the launch-argument box for the float32 one- and two-element Zhou path
    if constexpr (sizeof(T) == 4 && !Pol::species_addresses)
        if (S.boxed) return eam_dispatch_lpa<T, Pol, 2>(lpa, S, nl, P, E, rc2, B, ck, so, cs, n_chunks, phases, st);
    return S.ortho ? eam_dispatch_lpa<T, Pol, 1>(lpa, S, nl, P, E, rc2, B, ck, so, cs, n_chunks, phases, st)
                   : eam_dispatch_lpa<T, Pol, 0>(lpa, S, nl, P, E, rc2, B, ck, so, cs, n_chunks, phases, st);
}

// The constants of the one- and two-element Zhou path from the host copies
// of the tables; false when the tables have none, are not a fused Zhou set
// or have more than two elements.  The element parameters are those of each
// density row (ZHOU_KEYS order: r_e f_e rho_e rho_s alpha beta A B kappa
// lambda ...); the switch is the shared one of the table.
template <typename T>
static bool make_zk(const mbf_eam_tables *tab, ZK<T> &K) {
    if (!tab->zhou_fused || tab->ns < 1 || tab->ns > 2 || !tab->P_host || !tab->rho_f_host || !tab->phi_f_host)
        return false;
    const double LOG2E = 1.4426950408889634074;
    for (int s = 0; s < 2; ++s) {
        const double *p = tab->P_host + (size_t)tab->rho_f_host[s < tab->ns ? s : 0] * EAM_NCOL;
        const double re = p[0], fe = p[1], alpha = p[4], beta = p[5];
        ZEl<T> &q = K.el[s];
        q.ire = (T)(1.0 / re);
        q.re = (T)re;
        q.lam = (T)p[9];
        q.kap = (T)p[8];
        q.beta = (T)beta;
        q.alpha = (T)alpha;
        q.eb = (T)(-beta * LOG2E / re);
        q.ea = (T)(-alpha * LOG2E / re);
        if (!(fe > 0.0)) return false;
        q.fe = (T)fe;
        q.fe_ire = (T)(fe / re);
        q.lfe = (T)std::log2(fe);
        q.A = (T)p[6];
        q.B = (T)p[7];
    }
    const double *p0 = tab->P_host + (size_t)tab->rho_f_host[0] * EAM_NCOL;
    const double rc = p0[2 * EAM_NZ], w = p0[2 * EAM_NZ + 1];
    if (!(w > 0.0)) return false;
    K.r0 = (T)(rc - w);
    K.iw = (T)(1.0 / w);
    K.m30iw = (T)(-30.0 / w);
    double chi = 1.0;
    if (tab->ns == 2) chi = tab->P_host[(size_t)tab->phi_f_host[1] * EAM_NCOL + 2 * EAM_NZ + 2];
    K.half_chi = (T)(0.5 * chi);
    return true;
}

template <typename T>
static int eam_select(const mbf_eam_tables *tab, int lpa, const SysView &S, const mbf_nlist *nl, const EamDev &E,
                      double rc2, const EamBufs &B, Chk ck, const SiteOut &so, const ChunkSums &cs, int n_chunks,
                      int ph, cudaStream_t st) {
    ZK<T> K;
    if (make_zk<T>(tab, K)) {
        if (tab->ns == 1)
            return eam_dispatch<T>(PolZ2<T, 1>{K}, lpa, S, nl, E, rc2, B, ck, so, cs, n_chunks, ph, st);
        if constexpr (sizeof(T) == 4) {
            ZK2x X;
            make_zk2x(K, X);
            return eam_dispatch<T>(PolZ2x{K, X}, lpa, S, nl, E, rc2, B, ck, so, cs, n_chunks, ph, st);
        } else {
            return eam_dispatch<T>(PolZ2<T, 2>{K}, lpa, S, nl, E, rc2, B, ck, so, cs, n_chunks, ph, st);
        }
    }
    if (tab->zhou_fused != 0 && tab->ns <= EAM_MAXSP)
        return eam_dispatch<T>(PolZSmem<T>{E}, lpa, S, nl, E, rc2, B, ck, so, cs, n_chunks, ph, st);
    return eam_dispatch<T>(PolGeneric<T>{E}, lpa, S, nl, E, rc2, B, ck, so, cs, n_chunks, ph, st);
}

}  // namespace mbf

using namespace mbf;

// The evaluation's phases (PH_*): with PH_EMBED alone F'(rho-bar) of every
// atom is copied to fprime_out; with PH_FORCE alone fprime_in replaces F'
// before the force pass (the workspace must hold the same list's embedding
// pass); both: the whole evaluation.
static int eam_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                    const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                    size_t workspace_bytes, double *forces, double *energy, double *virial, const SiteOut &so,
                    void *stream, int phases = PH_ALL, double *fprime_out = nullptr,
                    const double *fprime_in = nullptr) {
    if (!sys || !nl || !tab || !plan || !workspace) return MBF_ERR_ARGUMENT;
    if ((phases & PH_FORCE) && (!forces || !energy || !virial)) return MBF_ERR_ARGUMENT;
    if (phases == PH_EMBED && !fprime_out) return MBF_ERR_ARGUMENT;
    if (phases == PH_FORCE && !fprime_in) return MBF_ERR_ARGUMENT;
    if (precision != MBF_FP64 && precision != MBF_MIXED) return MBF_ERR_ARGUMENT;
    if (nl->n_atoms != sys->n_atoms || tab->ns <= 0 || sys->n_struct <= 0) return MBF_ERR_ARGUMENT;
    if (nl->n_slots < 0 || nl->n_slots > 0x7fffff00LL) return MBF_ERR_ARGUMENT;
    // the per-structure completion counters live in a region of n_chunks
    // words; every structure owns at least one chunk
    if (plan->n_chunks <= 0 || plan->n_chunks < sys->n_struct) return MBF_ERR_ARGUMENT;
    const int lpa = lanes_per_atom > 0 ? lanes_per_atom : 8;
    if (lpa != 1 && lpa != 2 && lpa != 4 && lpa != 8) return MBF_ERR_ARGUMENT;
    EvalLayout L = eval_layout(sys->n_atoms, nl->n_slots, plan->n_chunks);
    if (workspace_bytes < L.total) return MBF_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    Chk ck;
    ck.err = ws_at<int>(workspace, L.err);
    ck.n_atoms = sys->n_atoms;
    ck.n_slots = (int)nl->n_slots;
    ck.ns = tab->ns;
    if ((phases & PH_EMBED) && cudaMemsetAsync(ck.err, 0, ERR_CLEAR_BYTES, st) != cudaSuccess) return MBF_ERR_CUDA;
    if (sys->n_atoms == 0) {
        if (!(phases & PH_FORCE)) return MBF_OK;
        if (cudaMemsetAsync(energy, 0, sizeof(double) * sys->n_struct, st) != cudaSuccess) return MBF_ERR_CUDA;
        if (cudaMemsetAsync(virial, 0, sizeof(double) * 9 * sys->n_struct, st) != cudaSuccess) return MBF_ERR_CUDA;
        return MBF_OK;
    }
    if (!nl->upper || !nl->row_off || !nl->nbr || !nl->rev) return MBF_ERR_ARGUMENT;
    SysView S = make_view(sys);
    // one diagonal cell known on the host: its lengths travel with the
    // launch -- not inside a stream capture, whose graph must read the
    // device cell at each replay (the lattice may change between replays)
    if (sys->n_struct == 1 && sys->orthorhombic && sys->cells_host) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        const cudaError_t qe = cudaStreamIsCapturing(st, &cap);
        if (qe != cudaSuccess) (void)cudaGetLastError();  // not a launch error: keep the cell in memory
        if (qe == cudaSuccess && cap == cudaStreamCaptureStatusNone) {
            const double *c = sys->cells_host;
            S.boxed = 1;
            S.box[0] = c[0];
            S.box[1] = c[4];
            S.box[2] = c[8];
            S.box[3] = c[9];
            S.box[4] = c[13];
            S.box[5] = c[17];
        }
    }
    EamDev E;
    E.ns = tab->ns; E.nf = tab->nf; E.nX = tab->nX;
    E.codes = tab->codes; E.P = tab->P; E.xo = tab->xo; E.nx = tab->nx;
    E.X = tab->X; E.C = tab->C;
    E.rho_f = tab->rho_f; E.F_f = tab->F_f; E.phi_f = tab->phi_f;
    E.r_cut = tab->r_cut;
    EamBufs B;
    B.pk = ws_at<double4>(workspace, L.pack);
    B.aux = ws_at<double>(workspace, L.atom_aux);
    B.slot = ws_at<char>(workspace, L.slot);
    B.f_local = ws_at<double>(workspace, L.f_local);
    B.forces = forces;
    B.per_atom = ws_at<double>(workspace, L.per_atom);
    ChunkSums cs = {plan->chunk, plan->chunk_first, B.per_atom, ws_at<double>(workspace, L.partial), energy, virial,
                    ws_at<unsigned>(workspace, L.sdone)};
    const size_t n = (size_t)sys->n_atoms;
    if (phases & PH_FORCE) {
        if (cudaMemsetAsync(cs.sdone, 0, sizeof(unsigned) * (size_t)sys->n_struct, st) != cudaSuccess)
            return MBF_ERR_CUDA;
        // F' of every atom into the records the force pass gathers (column 3
        // of pk, column 0 of aux), strided copies on the stream
        if (!(phases & PH_EMBED) &&
            (cudaMemcpy2DAsync(reinterpret_cast<double *>(B.pk) + 3, sizeof(double4), fprime_in, sizeof(double),
                               sizeof(double), n, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
             cudaMemcpy2DAsync(B.aux, 2 * sizeof(double), fprime_in, sizeof(double), sizeof(double), n,
                               cudaMemcpyDeviceToDevice, st) != cudaSuccess))
            return MBF_ERR_CUDA;
    }
    const double rc2 = tab->r_cut * tab->r_cut;
    int rc = precision == MBF_FP64
                 ? eam_select<double>(tab, lpa, S, nl, E, rc2, B, ck, so, cs, plan->n_chunks, phases, st)
                 : eam_select<float>(tab, lpa, S, nl, E, rc2, B, ck, so, cs, plan->n_chunks, phases, st);
    if (rc != MBF_OK || phases != PH_EMBED) return rc;
    if (cudaMemcpy2DAsync(fprime_out, sizeof(double), B.aux, 2 * sizeof(double), sizeof(double), n,
                          cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return MBF_ERR_CUDA;
    return MBF_OK;
}

extern "C" int mbf_eam_embedding(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                                 const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                                 size_t workspace_bytes, double *fprime, void *stream) {
    SiteOut none = {nullptr, nullptr, nullptr};
    return eam_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, nullptr, nullptr,
                    nullptr, none, stream, PH_EMBED, fprime, nullptr);
}

extern "C" int mbf_eam_forces(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                              const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                              size_t workspace_bytes, const double *fprime, double *forces, double *energy,
                              double *virial, void *stream) {
    SiteOut none = {nullptr, nullptr, nullptr};
    return eam_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, workspace_bytes, forces, energy,
                    virial, none, stream, PH_FORCE, nullptr, fprime);
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

// Device address of g_eam_scratch, looked up once per device (with that
// device current) and kept for the life of the process.  Host code must not
// use the array's name as a pointer: on the host it is only a stand-in
// symbol, not a device address.  The cached address belongs to the device's
// primary context, so a cudaDeviceReset() in the process invalidates it:
// callers of the no-allocation entry must not reset the device.
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
    if (!sys || !nl || !plan) return MBF_ERR_ARGUMENT;
    if (nl->n_slots < 0 || plan->n_chunks <= 0) return MBF_ERR_ARGUMENT;
    if (eval_layout(sys->n_atoms, nl->n_slots, plan->n_chunks).total > (size_t)MBF_STATIC_SCRATCH_BYTES)
        return MBF_ERR_SCRATCH_LIMIT;
    void *workspace = nullptr;
    int rc = scratch_address(&workspace);
    if (rc != MBF_OK) return rc;
    // the array keeps the previous call's contents: eam_eval clears the
    // error words and the completion counters at its start; every other
    // region is written before it is read
    SiteOut none = {nullptr, nullptr, nullptr};
    return eam_eval(sys, nl, tab, plan, precision, lanes_per_atom, workspace, MBF_STATIC_SCRATCH_BYTES, forces,
                    energy, virial, none, stream);
}

extern "C" int mbf_eam_eval_static_status(int *host_words, void *stream) {
    if (!host_words) return MBF_ERR_ARGUMENT;
    void *workspace = nullptr;
    int rc = scratch_address(&workspace);
    if (rc != MBF_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(host_words, workspace, 4 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MBF_ERR_CUDA;
    return MBF_OK;
}
