// Host launchers shared by the Wide-Fibonacci prover (prover.cu) and the
// stand-alone trait entry points (pcs_ops.cu), so that both run the same
// kernels for OODS sampling / eval_at_point and for grinding.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"

namespace stwo_b200 {

// Partial sums per polynomial of launch_poly_eval (its d_partial holds
// n_polys * poly_eval_chunks(lg) values).
uint32_t poly_eval_chunks(uint32_t lg);
// Low index bits h of the weight tables for polynomials of 2^lg
// coefficients: w_j = w_hi[j >> h] * w_lo[j & (2^h - 1)].
uint32_t poly_eval_lo_bits(uint32_t lg);
// Values at one point of n_polys (<= 1024) polynomials of 2^lg natural-order
// coefficients each, from the weight tables of launch_eval_weights (w_lo:
// 2^h entries, w_hi: 2^(lg - h), h = poly_eval_lo_bits(lg)):
// d_out[p] = sum_j coeff_p[j] w_j.
int launch_poly_eval(const uint32_t* const* polys, uint32_t n_polys, uint32_t lg, const qm31* d_w_lo,
                     const qm31* d_w_hi, qm31* d_partial, qm31* d_out, cudaStream_t s, char* err, size_t err_len);
// Weight tables of the point z for polynomials of 2^lg coefficients.
int launch_eval_weights(const spoint& z, uint32_t lg, qm31* d_w_lo, qm31* d_w_hi, cudaStream_t s, char* err,
                        size_t err_len);
// One proof-of-work batch: nonces (hi << 32) | (low_base + t), t < count
// (a multiple of 256), prefixed digest `pre`; the smallest hit is
// atomicMin'ed into *d_found.
int launch_grind(const uint32_t pre[8], uint32_t hi, uint32_t low_base, uint32_t count, uint32_t bits, int m31,
                 uint32_t* d_found, cudaStream_t s, char* err, size_t err_len);

}  // namespace stwo_b200
