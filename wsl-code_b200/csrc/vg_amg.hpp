// Smoothed-aggregation algebraic multigrid for the pressure Schur block of the k = 0 saddle point
// system, S = W diag(A)^{-1} W^T (a cell-graph Laplacian with weights 1/diag(A) on the edges).
//
// The reference preconditions with a PETSc ILU(0) on the CPU or, matrix-free, with the diagonal
// |rate M| + sum W^2/d (vem/CurvedVEM_Darcy_gpu/src/krylov.cu:99-117, src/equation_gpu.cu:282-315),
// which its own notes call weak for large meshes. Here the pressure block of the SPD block-diagonal
// MINRES preconditioner is one symmetric V-cycle on S (Jacobi pre- and post-smoothing with the same
// weight, exact coarsest solve), built on the host once per operator and applied on the device.
#pragma once
#include <vector>

#include "vg_common.cuh"

namespace vg {

struct HostCsr {
    int n = 0, m = 0;  // rows, columns
    std::vector<int> ptr, col;
    std::vector<double> val;
};

// sliced ELL with slice height 32: entry k of row r lives at soff[r / 32] + k * 32 + r % 32,
// padding entries have col = 0 and val = 0
template <typename T>
struct DevSell {
    int n = 0, nslices = 0;
    const long long* soff = nullptr;
    const int* width = nullptr;
    const int* col = nullptr;
    const T* val = nullptr;
};

// CSR for the rectangular transfer operators and the coarse Galerkin operators, processed in row
// blocks: block b covers rows [rb[b].x, rb[b + 1].x) and entries [rb[b].y, rb[b + 1].y)
template <typename T>
struct DevCsr {
    int n = 0, nblk = 0;
    int slots = 1;  // CTAs of the kernel resident at once on the device (grid cap)
    const int2* rb = nullptr;
    int* err = nullptr;  // set to 1 when a staged copy never lands (never in a correct run)
    const int* ptr = nullptr;
    const int* col = nullptr;
    const T* val = nullptr;
};

// coarsest level: at most this many rows, inverted densely (2500^2 doubles = 50 MB)
constexpr int COARSE_MAX = 2500;
// largest coarsest level accepted when coarsening stops early (level cap)
constexpr int DENSE_MAX = 4096;

class Amg {
public:
    // build the hierarchy of S (host CSR, symmetric positive definite or semi-definite); first_P, when
    // given, is the prolongator of the finest level (no aggregation there); fine_order, when given,
    // renumbers the finest level's rows for the vectors the cycle acts on (row i -> fine_order[i])
    // after S has been coarsened in its own order
    void setup(const HostCsr& S, const HostCsr* first_P, const std::vector<int>* fine_order = nullptr);
    bool ready() const { return !levels_.empty(); }
    int levels() const { return int(levels_.size()); }
    long long nnz() const;
    // z = V-cycle(b) on the device (b, z of length n0); FP64 or FP32 copy of the hierarchy
    void vcycle(const double* b, double* z, cudaStream_t s);
    void vcycle(const float* b, float* z, cudaStream_t s);
    long long launches = 0;
    // true when a cycle kernel gave up on a copy (the flag is cleared)
    bool failed();
    // Recompute every value of the hierarchy on the device for a new finest-level operator with the
    // same sparsity: the aggregates, sparsity patterns and smoothing weights of setup() are kept
    // (a valid multigrid for any values; the captured cycle's device addresses do not change).
    // a0: the finest level's values in the order of its stored pattern (level0_ptr / level0_col).
    void refresh(const double* a0);
    const int* level0_ptr() const { return levels_.empty() ? nullptr : levels_[0].dpa_ptr.data(); }
    const int* level0_col() const { return levels_.empty() ? nullptr : levels_[0].dpa_col.data(); }
    long long level0_nnz() const { return levels_.empty() ? 0 : (long long)levels_[0].pa_col.size(); }

private:
    struct Sell {
        int n = 0, nslices = 0;
        std::vector<long long> soff;
        std::vector<int> width, col;
        std::vector<double> val;
        // CSR copy used instead of the slices when rows are long
        bool csr = false;
        std::vector<int> cptr, ccol;
        std::vector<int> rb;  // row blocks: (first row, first entry) pairs, one past the last block included
        std::vector<double> cval;
    };
    struct Level {
        int n = 0, nc = 0;
        double omega = 0;
        Sell A, P, R;  // P: n x nc, R = P^T: nc x n (absent on the coarsest level)
        std::vector<double> dinv;
        // structure kept for refresh(): stored CSR pattern of A, aggregate of every stored row (empty
        // when the prolongator is given), position in P of every R entry, SELL slot of every CSR
        // entry of A (SELL storage)
        std::vector<int> pa_ptr, pa_col, agg, r2p;
        std::vector<long long> sellpos;
        bool fixedP = false;
        DevBuf<int> dpa_ptr, dpa_col, dagg, dr2p;
        DevBuf<long long> dsellpos;
        // device
        DevBuf<long long> dA_soff, dP_soff, dR_soff;
        DevBuf<int> dA_w, dA_col, dP_w, dP_col, dR_w, dR_col;
        DevBuf<int> cA_ptr, cA_col, cP_ptr, cP_col, cR_ptr, cR_col, cA_rb, cP_rb, cR_rb;
        DevBuf<double> cA_v64, cP_v64, cR_v64;
        DevBuf<float> cA_v32, cP_v32, cR_v32;
        DevBuf<double> dA_v64, dP_v64, dR_v64, dinv64, x64, b64, r64, t64;
        DevBuf<float> dA_v32, dP_v32, dR_v32, dinv32, x32, b32, r32, t32;
    };
    template <typename T>
    void cycle(int l, const T* b, T* z, cudaStream_t s);
    void dense_inverse_device(const std::vector<double>& a, int n);
    void dense_inverse_of(double* d, int n);  // in-place device matrix -> dinvc64_ / dinvc32_
    template <typename T>
    DevSell<T> view(const Level& L, int which) const;
    template <typename T>
    DevCsr<T> cview(const Level& L, int which) const;

    std::vector<Level> levels_;
    int ncoarse_ = 0;
    DevBuf<int> err_;
    int csr_slots_[2] = {1, 1};  // resident CTAs of the CSR kernels on this hierarchy's device (FP32, FP64)
    DevBuf<double> dinvc64_;  // dense inverse of the coarsest matrix
    DevBuf<float> dinvc32_;
};

}  // namespace vg
