// Matrix-free apply: argument block and launcher.
#pragma once
#include <vector>

#include "vg_common.cuh"

namespace vg {

template <typename T>
struct ApplyArgs {
    const T* x;
    T* y;               // flux edge entries must be zero on entry (atomic scatter)
    const T* A;         // packed A_E, piece layout
    const T* W;         // W_E (k >= 1), piece layout
    const int* map;     // signed flux dof map, piece layout
    const int* slot_cell;
    const Piece* pieces;
    int npieces, k;
    const T* L;         // multiplier vector per cell (q), when mult
    const int* mask;    // essential-BC mask (N), when constrained
    const int* flags;   // optional: skip when flags[0] != 0
    long long nf, N;
    T psign;
    int constrained, mult;
    double* partials;   // 2 per block, when red or mult
    unsigned int* counter;
    double* red;        // optional: quadratic form x^T K x -> red[0]
    int total_blocks, block_off;
};

constexpr int APPLY_THREADS = 256;
int apply_blocks(int npieces);

template <typename T>
void launch_apply(ApplyArgs<T> a, cudaStream_t s);

}  // namespace vg
