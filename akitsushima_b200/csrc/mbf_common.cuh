// Shared device helpers of the many-body force kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mbforce.h"

#define MBF_WARP 32
#define MBF_FULL 0xffffffffu

// Device error word bits (workspace word 0 of each call's error block).
#define MBF_DEV_ROW_TOO_LONG 1
#define MBF_DEV_BAD_INDEX 2

#define MBF_CHECK_LAUNCH()                                   \
    do {                                                     \
        if (cudaGetLastError() != cudaSuccess) return MBF_ERR_CUDA; \
    } while (0)

namespace mbf {

// Device view of mbf_system.
struct SysView {
    int n_atoms;
    int n_struct;
    const double *pos;
    const int *types;
    const int *atom_struct;
    const int *struct_off;
    const double *cells;
    int ortho;
    int boxed;      // 1: one diagonal cell, its lengths and inverses in box
    double box[6];  // L0 L1 L2 1/L0 1/L1 1/L2 (only with boxed)
};

static inline SysView make_view(const mbf_system *s) {
    SysView v;
    v.n_atoms = s->n_atoms;
    v.n_struct = s->n_struct;
    v.pos = s->positions;
    v.types = s->types;
    v.atom_struct = s->atom_struct;
    v.struct_off = s->struct_off;
    v.cells = s->cells;
    v.ortho = s->orthorhombic;
    v.boxed = 0;
    for (int k = 0; k < 6; ++k) v.box[k] = 0.0;
    return v;
}

// Round half to even for |x| < 2^51 by the 1.5 * 2^52 shift: the sum's
// spacing is exactly 1, so the add rounds x to the nearest integer (ties to
// even) and the subtraction is exact.  Equal to rint(x) there, and cheaper
// than the conversion unit's rounding.
__device__ __forceinline__ double rint_shift(double x) {
    const double M = 6755399441055744.0;
    return __dsub_rn(__dadd_rn(x, M), M);
}

// Minimum-image displacement of r = (rx, ry, rz) in the cell `c` (lattice
// rows c[0..8], inverse c[9..17]) evaluated exactly as the reference's
// neighbour-list kernel does (engine/neighborlist.py:350-362): each dot
// product summed left to right, no fused multiply-add, s -= rint(s) with
// round-half-even.  The intrinsics pin the rounding of every operation.
__device__ __forceinline__ void mic_exact(const double *__restrict__ c, double rx,
                                          double ry, double rz, double &dx,
                                          double &dy, double &dz) {
    const double *inv = c + 9;
    double sx = __dadd_rn(__dadd_rn(__dmul_rn(rx, __ldg(inv + 0)), __dmul_rn(ry, __ldg(inv + 3))),
                          __dmul_rn(rz, __ldg(inv + 6)));
    double sy = __dadd_rn(__dadd_rn(__dmul_rn(rx, __ldg(inv + 1)), __dmul_rn(ry, __ldg(inv + 4))),
                          __dmul_rn(rz, __ldg(inv + 7)));
    double sz = __dadd_rn(__dadd_rn(__dmul_rn(rx, __ldg(inv + 2)), __dmul_rn(ry, __ldg(inv + 5))),
                          __dmul_rn(rz, __ldg(inv + 8)));
    sx = __dsub_rn(sx, rint_shift(sx));
    sy = __dsub_rn(sy, rint_shift(sy));
    sz = __dsub_rn(sz, rint_shift(sz));
    dx = __dadd_rn(__dadd_rn(__dmul_rn(sx, __ldg(c + 0)), __dmul_rn(sy, __ldg(c + 3))),
                   __dmul_rn(sz, __ldg(c + 6)));
    dy = __dadd_rn(__dadd_rn(__dmul_rn(sx, __ldg(c + 1)), __dmul_rn(sy, __ldg(c + 4))),
                   __dmul_rn(sz, __ldg(c + 7)));
    dz = __dadd_rn(__dadd_rn(__dmul_rn(sx, __ldg(c + 2)), __dmul_rn(sy, __ldg(c + 5))),
                   __dmul_rn(sz, __ldg(c + 8)));
}

__device__ __forceinline__ double r2_exact(double dx, double dy, double dz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Displacement r_b - r_a (minimum image) of two atoms of one structure.
__device__ __forceinline__ void pair_vec(const SysView &S, const double *__restrict__ cell,
                                         int a, int b, double &dx, double &dy, double &dz) {
    const double *pa = S.pos + 3 * (size_t)a;
    const double *pb = S.pos + 3 * (size_t)b;
    mic_exact(cell, __ldg(pb) - __ldg(pa), __ldg(pb + 1) - __ldg(pa + 1),
              __ldg(pb + 2) - __ldg(pa + 2), dx, dy, dz);
}

__device__ __forceinline__ const double *cell_of(const SysView &S, int atom) {
    int s = S.n_struct > 1 ? __ldg(S.atom_struct + atom) : 0;
    return S.cells + 18 * (size_t)s;
}

// Sum over the LPA lanes of a lane group (all 32 lanes must call it).
template <int LPA, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int o = LPA / 2; o > 0; o >>= 1) v += __shfl_xor_sync(MBF_FULL, v, o, LPA);
    return v;
}

// Real-type helpers for templated float/double arithmetic.
template <typename T> struct RT;
template <> struct RT<double> {
    static __device__ __forceinline__ double ex(double x) { return exp(x); }
    static __device__ __forceinline__ double sn(double x) { return sin(x); }
    static __device__ __forceinline__ double cs(double x) { return cos(x); }
    static __device__ __forceinline__ double pw(double x, double y) { return pow(x, y); }
    static __device__ __forceinline__ double lg(double x) { return log(x); }
    static __device__ __forceinline__ double sq(double x) { return sqrt(x); }
};
template <> struct RT<float> {
    static __device__ __forceinline__ float ex(float x) { return expf(x); }
    static __device__ __forceinline__ float sn(float x) { return sinf(x); }
    static __device__ __forceinline__ float cs(float x) { return cosf(x); }
    static __device__ __forceinline__ float pw(float x, float y) { return powf(x, y); }
    static __device__ __forceinline__ float lg(float x) { return logf(x); }
    static __device__ __forceinline__ float sq(float x) { return sqrtf(x); }
};

// Exponential clamped at +-500 (reference engine/_numba_common.py:12-33).
// In float the upper branch saturates at FLT_MAX-range, which no physical
// bond reaches; the lower branch returns 0 as the reference does.
template <typename T>
__device__ __forceinline__ T clamped_exp(T x) {
    if (x > T(500)) return RT<T>::ex(T(500));
    if (x < T(-500)) return T(0);
    return RT<T>::ex(x);
}

// Division: IEEE in float64; the fast approximate quotient (2 ulp) in
// float32, whose callers are the mixed-precision terms only.
template <typename T> __device__ __forceinline__ T fdiv(T a, T b);
template <> __device__ __forceinline__ double fdiv<double>(double a, double b) { return a / b; }
template <> __device__ __forceinline__ float fdiv<float>(float a, float b) { return __fdividef(a, b); }

// Integer power by repeated multiplication for the small fixed exponents
// used by the potentials.
template <typename T>
__device__ __forceinline__ T pow20(T u, T &u19) {
    T u2 = u * u, u4 = u2 * u2, u8 = u4 * u4, u16 = u8 * u8;
    u19 = u16 * u2 * u;
    return u16 * u4;
}

// Grid size for persistent grid-stride kernels.
int persistent_grid(int blocks_needed, int block, const void *kernel, size_t smem = 0);

}  // namespace mbf
