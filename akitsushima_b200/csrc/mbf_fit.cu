// The fit loss over a batch and its gradient with respect to the batch's
// energies, forces and virials, on the device.
//
// Replaces the per-structure loss loop of fitting/loss.py:184-260 (squared
// or Huber, per-structure trust weight and scale): for structure s with
// n_s original atoms (evaluated as a supercell of k_s replicas when its
// cell is thin),
//   e_sq = (E_s / k_s - n_s e_ref)^2
//   f_sq = r0^2 sum_a |F_a - F_ref,a|^2 / (3 n_s)      (original atoms)
//   s_sq = (V_s eps0)^2 mean_9 (W_s / V_sup,s - sigma_ref)^2
//   loss = sum_s cw_s [w_E h(e_sq) + w_F h(f_sq) [forces] + w_S h(s_sq) [stress]]
// with h the identity or the Huber map of the squared residual
// (fitting/loss.py:29-48).  The same pass writes d loss / dE, dF, dW, the
// upstream gradients the adjoint kernels take.  Sums run in a fixed order.
#include "mbf_util.cuh"

namespace mbf {

// Huber map of a squared residual and its derivative in the square.
__device__ __forceinline__ void huber_sq(double sq, double delta, int huber, double &h, double &dh) {
    if (!huber) {
        h = sq;
        dh = 1.0;
        return;
    }
    double r = sqrt(sq > 1e-300 ? sq : 1e-300);
    if (r <= delta) {
        h = sq;
        dh = 1.0;
    } else {
        h = 2.0 * delta * r - delta * delta;
        dh = delta / r;
    }
}

// Warp per structure: the force residual sum over its original atoms (lane
// strided, fixed tree), then lane 0 the structure's loss terms, dloss/dE_s,
// dloss/dW_s and the factor of dloss/dF_a.
__global__ void fit_struct_terms(mbf_fit_set P, const double *__restrict__ E, const double *__restrict__ F,
                                 const double *__restrict__ W, double *__restrict__ per, double *__restrict__ gE,
                                 double *__restrict__ gW, double *__restrict__ fac) {
    int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
    if (s >= P.n_struct) return;  // whole warps leave together
    int a0 = P.struct_off[s], n = P.n_orig[s], fo = P.fref_off[s];
    bool has_f = P.fmask[s] != 0.0, has_s = P.smask[s] != 0.0;
    double acc = 0.0;
    if (has_f)
        for (int a = l; a < n; a += 32) {
            const double *f = F + 3 * (size_t)(a0 + a);
            const double *r = P.f_ref + 3 * (size_t)(fo + a);
            double dx = f[0] - r[0], dy = f[1] - r[1], dz = f[2] - r[2];
            acc += dx * dx + dy * dy + dz * dz;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MBF_FULL, acc, o);
    if (l != 0) return;
    double cw = P.cw[s], inv_k = P.inv_k[s], nn = (double)n;
    double de = E[s] * inv_k - nn * P.e_ref[s];
    double hE, dhE, hF, dhF, hS, dhS;
    huber_sq(de * de, P.delta_e, P.huber, hE, dhE);
    double fq = n > 0 ? P.r0 * P.r0 * acc / (3.0 * nn) : 0.0;
    huber_sq(fq, P.delta_f, P.huber, hF, dhF);
    double ds[9], sq = 0.0, vs = P.vsup[s];
    for (int k = 0; k < 9; ++k) {
        ds[k] = W[9 * (size_t)s + k] / vs - P.s_ref[9 * (size_t)s + k];
        sq += ds[k] * ds[k];
    }
    double ve = P.vol[s] * P.eps0;
    huber_sq(ve * ve * sq / 9.0, P.delta_s, P.huber, hS, dhS);
    per[s] = cw * (P.w_e * hE + (has_f ? P.w_f * hF : 0.0) + (has_s ? P.w_s * hS : 0.0));
    gE[s] = cw * P.w_e * dhE * 2.0 * de * inv_k;
    fac[s] = (has_f && n > 0) ? cw * P.w_f * dhF * P.r0 * P.r0 * 2.0 / (3.0 * nn) : 0.0;
    double gs = has_s ? cw * P.w_s * dhS * ve * ve * (2.0 / 9.0) / vs : 0.0;
    for (int k = 0; k < 9; ++k) gW[9 * (size_t)s + k] = gs * ds[k];
}

// dloss/dF per atom (0 for the replicas of a thin cell); block 0's first
// warp also sums the per-structure terms into the loss (fixed order).
__global__ void fit_atom_grad(mbf_fit_set P, const double *__restrict__ F, const double *__restrict__ fac,
                              const double *__restrict__ per, double *__restrict__ gF, double *__restrict__ loss) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < P.n_atoms) {
        int s = P.atom_struct[a];
        int la = a - P.struct_off[s];
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        if (la < P.n_orig[s] && fac[s] != 0.0) {
            const double *r = P.f_ref + 3 * (size_t)(P.fref_off[s] + la);
            double c = fac[s];
            g0 = c * (F[3 * (size_t)a] - r[0]);
            g1 = c * (F[3 * (size_t)a + 1] - r[1]);
            g2 = c * (F[3 * (size_t)a + 2] - r[2]);
        }
        gF[3 * (size_t)a] = g0;
        gF[3 * (size_t)a + 1] = g1;
        gF[3 * (size_t)a + 2] = g2;
    }
    if (blockIdx.x == 0 && threadIdx.x < 32) {
        double acc = 0.0;
        for (int s = threadIdx.x; s < P.n_struct; s += 32) acc += per[s];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(MBF_FULL, acc, o);
        if (threadIdx.x == 0) *loss = acc;
    }
}

}  // namespace mbf

using namespace mbf;

extern "C" {

size_t mbf_fit_loss_workspace_bytes(int n_struct) {
    if (n_struct < 0) return 0;
    return 2 * align256(sizeof(double) * (size_t)(n_struct > 0 ? n_struct : 1));
}

int mbf_fit_loss(const mbf_fit_set *set, const double *energy, const double *forces, const double *virial,
                 void *workspace, size_t workspace_bytes, double *loss, double *g_energy, double *g_forces,
                 double *g_virial, void *stream) {
    if (!set || !energy || !forces || !virial || !workspace || !loss || !g_energy || !g_forces || !g_virial)
        return MBF_ERR_ARGUMENT;
    if (set->n_struct <= 0 || set->n_atoms < 0) return MBF_ERR_ARGUMENT;
    if (!set->struct_off || !set->atom_struct || !set->n_orig || !set->fref_off || !set->inv_k || !set->e_ref ||
        !set->f_ref || !set->s_ref || !set->vol || !set->vsup || !set->fmask || !set->smask || !set->cw)
        return MBF_ERR_ARGUMENT;
    if (workspace_bytes < mbf_fit_loss_workspace_bytes(set->n_struct)) return MBF_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    double *per = ws_at<double>(workspace, 0);
    double *fac = ws_at<double>(workspace, align256(sizeof(double) * (size_t)set->n_struct));
    fit_struct_terms<<<(set->n_struct * 32 + 127) / 128, 128, 0, st>>>(*set, energy, forces, virial, per, g_energy,
                                                                       g_virial, fac);
    MBF_CHECK_LAUNCH();
    int blocks = set->n_atoms > 0 ? (set->n_atoms + 255) / 256 : 1;
    fit_atom_grad<<<blocks, 256, 0, st>>>(*set, forces, fac, per, g_forces, loss);
    MBF_CHECK_LAUNCH();
    return MBF_OK;
}

}  // extern "C"
