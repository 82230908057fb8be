// Pieces of the AmplitudePhase / NGDExact path (ap.cu) that live next to the
// Hamiltonian kernels.
#pragma once
#include "internal.hpp"

namespace yq {

// out(k) = sum_j H_sub(k, j) psi(j) over a basis closed under H, with
// H_sub(k, j) = column(basis[k])[basis[j]] (ED/ConstructSparseMat.hpp:31-56):
// the diagonal of configuration k times psi(k) plus every off-diagonal request
// of the state form at configuration k times psi at the flipped configuration.
// Requests that leave the basis are dropped.
void ham_apply_basis(yq_ham_s* H, uint64_t dim, int kind, int nup, const uint64_t* d_binom, const uint64_t* d_index,
                     const int8_t* d_sigma, const c128* d_psi, c128* d_out, cudaStream_t st);

}  // namespace yq
