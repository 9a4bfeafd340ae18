// eri_grad.cuh -- nuclear-coordinate gradient of the two-electron energy of
// a closed-shell density: the adjoint contraction of derivative ERIs with the
// density products, one kernel for every quartet class.
//
// With the half density P (P = C_occ C_occ^T, scfaux.c:24-41) the
// two-electron energy is E2 = tr(P G[P]) = sum_ijkl Gamma_ijkl (ij|kl) over
// ordered indices, and over the unique shell quartets with the degeneracy
// factor deg of the Fock kernels
//     Gamma_ijkl = 2 P_ij P_kl - (P_ik P_jl + P_il P_jk) / 2 .
// Open shell (spin densities Pa, Pb, the UHF energy of uhfscf.c:54-55 with
// G_s = J[Pa+Pb] - K[P_s]): with Pt = Pa + Pb
//     Gamma_ijkl = Pt_ij Pt_kl / 2 - sum_s (P_s,ik P_s,jl + P_s,il P_s,jk) / 4 .
// Its derivative with respect to the centre A of the first bra shell uses,
// per primitive of exponent alpha,
//     d phi_a / dA_x = 2 alpha phi_{a+1x} - a_x phi_{a-1x},
// i.e. one more unit of angular momentum in the 1-D Rys tables; centres B and
// C likewise; centre D by translational invariance, dD = -(dA + dB + dC).
// The Rys rule takes n = (L+1)/2 + 1 roots, exact for the raised integrals.
#pragma once
#include "eri.cuh"

namespace pg {

struct GradArgs {
    const int *ca, *cb;     // per shell pair: centre of the first and the second shell
    const double *ea;       // per primitive pair: exponent of the first shell's primitive
    double *grad;           // [ncen][3], accumulated with atomics
    int la, lb, lc, ld;     // quartet class in kernel orientation
};

// Launch the gradient kernel for the class in g over the quartets described
// by a (implicit or list mode, swap = 0; a.D0 = full n x n half density, or
// with a.D1 set the alpha and beta spin densities).
cudaError_t launch_eri_grad(const EriArgs &a, const GradArgs &g, cudaStream_t stream, int num_sms);

// Dynamic shared memory the class needs (bytes per block).
size_t eri_grad_smem(int la, int lb, int lc, int ld);

}  // namespace pg
