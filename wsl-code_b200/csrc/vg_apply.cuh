// Matrix-free apply: argument block, record-stream plan and launchers.
#pragma once
#include <vector>

#include "vg_common.cuh"

namespace vg {

// A run of consecutive piece records copied into one shared-memory stage by one bulk copy.
// bytes == 0 marks a piece too large for a stage: its cells read the operator from the
// strided global arrays instead.
struct ApplyBatch {
    long long off;  // byte offset of the first record in the stream
    int bytes;      // bytes of the run (multiple of 16)
    int first;      // first piece
    int count;      // pieces in the run
    int pad_[3];
};

template <typename T>
struct ApplyArgs {
    const T* x;
    T* y;               // flux edge entries must be zero on entry (atomic scatter)
    const T* A;         // packed A_E, piece layout
    const T* W;         // W_E (k >= 1), piece layout
    const int* map;     // signed flux dof map, piece layout (indices of the vectors' order)
    const int* prow;    // per slot: first pressure row of the cell (nf + rank * q), -1 on padding
    const Piece* pieces;
    int npieces, k;
    const T* L;         // multiplier vector, indexed like the pressure rows minus nf, when mult
    const int* mask;    // essential-BC mask (N), when constrained
    const int* flags;   // optional: skip when flags[0] != 0
    long long nf, N;
    T psign;
    int constrained, mult;
    double* partials;   // 2 per block, when red or mult
    unsigned int* counter;
    double* red;        // optional: quadratic form x^T K x -> red[0]
    // record stream (k <= 1): per piece one contiguous record
    //   int4 {ne, n, count, record bytes} | A_E (n(n+1)/2 x 32 T) | W_E (q n x 32 T, k >= 1)
    //   | map (n x 32 int) | pressure row (32 int)
    // streamed through a ring of shared-memory stages by cp.async.bulk; null: strided kernel
    const unsigned char* rec;
    const ApplyBatch* batches;
    const int* cta_batch;  // batches of CTA c: [cta_batch[c], cta_batch[c + 1])
    int ncta, stages, stage_bytes;
    int* err;              // set to 1 when a pipeline wait gives up (never in a correct run)
    int* stall;            // test hook: when nonzero, the first consumer to see it clears it and
                           // waits on a barrier nothing arrives on, so that its bounded wait runs out
};

constexpr int APPLY_THREADS = 256;
int apply_blocks(int npieces);

// Host plan of the record stream of one precision: record offsets, batches, CTA ranges.
struct StreamPlan {
    std::vector<long long> rec_off;  // npieces + 1 (bytes)
    std::vector<ApplyBatch> batches;
    std::vector<int> cta_batch;      // ncta + 1
    int stage_bytes = 0, stages = 0, ncta = 0;
    long long bytes = 0;
};
StreamPlan plan_stream(const std::vector<Piece>& pieces, int k, int elem_bytes, int sm_count);
// record bytes of one piece
long long record_bytes(const Piece& P, int k, int elem_bytes);

// write the records of all pieces (one warp per piece)
template <typename T>
void pack_stream(const Piece* pieces, int npieces, const long long* rec_off, const T* A, const T* W, const int* map,
                 const int* prow, int k, unsigned char* out, cudaStream_t s);
// raise the dynamic shared-memory limit of the streamed kernels (outside any stream capture)
void prepare_stream_kernels();

template <typename T>
void launch_apply(ApplyArgs<T> a, cudaStream_t s);

}  // namespace vg
