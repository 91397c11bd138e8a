// Host entry points of the FFT passes for the prover (fft.cu): an
// interpolation split into its passes, so that the first pass of a trace can
// run chunk by chunk while the rest of the trace is still arriving.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace stwo_b200 {

// Layers per pass of an n-layer transform, low layers first (the current plan).
std::vector<uint32_t> fft_split(uint32_t log_n);
// Pass `pi` of the in-place interpolation of n_cols columns of 2^log_n words
// under `split`; pass 0 over rows [row_begin, row_end) only (whole tiles of
// 2^split[0] consecutive rows), the later passes over every row.  Pass 0
// reads `src` instead of `cols` when given.
int interpolate_pass(uint32_t* const* cols, uint32_t n_cols, uint32_t log_n, const std::vector<uint32_t>& split,
                     uint32_t pi, uint64_t row_begin, uint64_t row_end, const uint32_t* d_itwiddles,
                     uint32_t tree_log_size, cudaStream_t s, char* err, size_t err_len,
                     const uint32_t* const* src = nullptr);
// The interpolation of n_cols columns of 2^log_n words in place (into the
// coefficients `coeffs`), from pass `first_pass` of `split` on, followed by
// their evaluation onto the 2^log_blowup times larger domain into `evals`
// (stwo_b200_interpolate_columns then stwo_b200_evaluate_polynomials, same
// words).  Where the split ends in a 10-layer strided pass over layers
// 10..19, 11..20 or 12..21 and the blowup is 1 or 2, that pass and the
// evaluation's first run as one kernel.  With first_pass 0 and src0 given, the first
// pass reads src0 (out of place).
int interpolate_evaluate(uint32_t* const* coeffs, uint32_t* const* evals, uint32_t n_cols, uint32_t log_n,
                         uint32_t log_blowup, const std::vector<uint32_t>& split, uint32_t first_pass,
                         const uint32_t* d_itwiddles, const uint32_t* d_twiddles, uint32_t tree_log_size,
                         cudaStream_t s, char* err, size_t err_len, const uint32_t* const* src0 = nullptr);

}  // namespace stwo_b200
