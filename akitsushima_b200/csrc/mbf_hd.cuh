// Hyper-dual arithmetic for the adjoint kernels: a number carries its value,
// one tangent (the direction of the upstream force and virial gradients)
// and K parameter directions with their tangent cross terms, so one
// evaluation of an energy term gives dV/dtheta_p and d(D_t V)/dtheta_p.
#pragma once

#include "mbf_util.cuh"

namespace mbf {

// v + t e + sum_p (p_p f_p + q_p e f_p): value, tangent, parameter
// derivatives and their tangent cross terms.
template <int K>
struct HD {
    double v, t, p[K], q[K];
};

template <int K>
__device__ __forceinline__ HD<K> hd_const(double v) {
    HD<K> r;
    r.v = v;
    r.t = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = r.q[k] = 0.0;
    return r;
}

// A parameter read at `site`: seeded if the site is one of this pass's.
template <int K>
__device__ __forceinline__ HD<K> hd_param(double v, int site, int first) {
    HD<K> r = hd_const<K>(v);
    int k = site - first;
#pragma unroll
    for (int q = 0; q < K; ++q)
        if (q == k) r.p[q] = 1.0;
    return r;
}

template <int K>
__device__ __forceinline__ HD<K> operator+(const HD<K> &a, const HD<K> &b) {
    HD<K> r;
    r.v = a.v + b.v;
    r.t = a.t + b.t;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r.p[k] = a.p[k] + b.p[k];
        r.q[k] = a.q[k] + b.q[k];
    }
    return r;
}

template <int K>
__device__ __forceinline__ HD<K> operator-(const HD<K> &a, const HD<K> &b) {
    HD<K> r;
    r.v = a.v - b.v;
    r.t = a.t - b.t;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r.p[k] = a.p[k] - b.p[k];
        r.q[k] = a.q[k] - b.q[k];
    }
    return r;
}

template <int K>
__device__ __forceinline__ HD<K> operator*(const HD<K> &a, const HD<K> &b) {
    HD<K> r;
    r.v = a.v * b.v;
    r.t = a.t * b.v + a.v * b.t;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r.p[k] = a.p[k] * b.v + a.v * b.p[k];
        r.q[k] = a.q[k] * b.v + a.p[k] * b.t + a.t * b.p[k] + a.v * b.q[k];
    }
    return r;
}

template <int K>
__device__ __forceinline__ HD<K> operator*(double s, const HD<K> &a) {
    HD<K> r;
    r.v = s * a.v;
    r.t = s * a.t;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r.p[k] = s * a.p[k];
        r.q[k] = s * a.q[k];
    }
    return r;
}

template <int K>
__device__ __forceinline__ HD<K> operator+(double s, const HD<K> &a) {
    HD<K> r = a;
    r.v += s;
    return r;
}

template <int K>
__device__ __forceinline__ HD<K> operator+(const HD<K> &a, double s) {
    HD<K> r = a;
    r.v += s;
    return r;
}

// f(a) from f, f', f'' at a.v (the chain rule to second, mixed order).
template <int K>
__device__ __forceinline__ HD<K> hd_apply(const HD<K> &a, double f, double f1, double f2) {
    HD<K> r;
    r.v = f;
    r.t = f1 * a.t;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        r.p[k] = f1 * a.p[k];
        r.q[k] = f1 * a.q[k] + f2 * a.t * a.p[k];
    }
    return r;
}

template <int K>
__device__ __forceinline__ HD<K> hd_inv(const HD<K> &a) {
    double i = 1.0 / a.v;
    return hd_apply<K>(a, i, -i * i, 2.0 * i * i * i);
}

template <int K>
__device__ __forceinline__ HD<K> operator/(const HD<K> &a, const HD<K> &b) {
    return a * hd_inv<K>(b);
}

template <int K>
__device__ __forceinline__ HD<K> hd_exp(const HD<K> &a) {
    double e = exp(a.v);
    return hd_apply<K>(a, e, e, e);
}

template <int K>
__device__ __forceinline__ HD<K> hd_log(const HD<K> &a) {
    double i = 1.0 / a.v;
    return hd_apply<K>(a, log(a.v), i, -i * i);
}

template <int K>
__device__ __forceinline__ HD<K> hd_sin(const HD<K> &a) {
    double s = sin(a.v), c = cos(a.v);
    return hd_apply<K>(a, s, c, -s);
}

// exp clamped as the reference's _nb_exp (engine/_numba_common.py:12-33):
// constant outside [-500, 500].
template <int K>
__device__ __forceinline__ HD<K> hd_cexp(const HD<K> &a) {
    if (a.v > 500.0) return hd_const<K>(exp(500.0));
    if (a.v < -500.0) return hd_const<K>(0.0);
    return hd_exp<K>(a);
}

template <int K>
__device__ __forceinline__ HD<K> hd_pow(const HD<K> &x, const HD<K> &y) {
    return hd_exp<K>(y * hd_log<K>(x));
}

// Upstream gradients of the adjoint entries.
struct AdjIn {
    const double *gE, *gF, *gW;  // (S,), (N, 3), (S, 9); null = 0
};

// Pair vector, its length and its tangent t = gF_i - gF_j - gW d.
__device__ __forceinline__ void adj_leg(const SysView &S, const AdjIn &G, const double *cell, int i, int j,
                                        int s_struct, double d[3], double &r, double tg[3]) {
    mic_exact(cell, S.pos[3 * (size_t)j] - S.pos[3 * (size_t)i], S.pos[3 * (size_t)j + 1] - S.pos[3 * (size_t)i + 1],
              S.pos[3 * (size_t)j + 2] - S.pos[3 * (size_t)i + 2], d[0], d[1], d[2]);
    r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int a = 0; a < 3; ++a) {
        double t = 0.0;
        if (G.gF) t = G.gF[3 * (size_t)i + a] - G.gF[3 * (size_t)j + a];
        if (G.gW) {
            const double *w = G.gW + 9 * (size_t)s_struct + 3 * a;
            t -= w[0] * d[0] + w[1] * d[1] + w[2] * d[2];
        }
        tg[a] = t;
    }
}

}  // namespace mbf
