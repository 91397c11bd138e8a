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
// 2^split[0] consecutive rows), the later passes over every row.
int interpolate_pass(uint32_t* const* cols, uint32_t n_cols, uint32_t log_n, const std::vector<uint32_t>& split,
                     uint32_t pi, uint64_t row_begin, uint64_t row_end, const uint32_t* d_itwiddles,
                     uint32_t tree_log_size, cudaStream_t s, char* err, size_t err_len);

}  // namespace stwo_b200
