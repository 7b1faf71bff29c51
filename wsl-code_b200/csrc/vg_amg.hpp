// Smoothed-aggregation algebraic multigrid for the pressure Schur block of the k = 0 saddle point
// system, S = W diag(A)^{-1} W^T (a cell-graph Laplacian with weights 1/diag(A) on the edges).
//
// The reference preconditions with a PETSc ILU(0) on the CPU or, matrix-free, with the diagonal
// |rate M| + sum W^2/d (vem/CurvedVEM_Darcy_gpu/src/krylov.cu:99-117, src/equation_gpu.cu:282-315),
// which its own notes call weak for large meshes. Here the pressure block of the SPD block-diagonal
// MINRES preconditioner is one symmetric V-cycle on S (Jacobi pre- and post-smoothing with the same
// weight, exact coarsest solve), built on the host once per operator and applied on the device.
//
// The cycle runs in a composite form with the same operator. With S_l = omega_l D_l^{-1}, one
// pre-smoothing step from zero, the residual, the restriction, the coarse correction and one
// post-smoothing step give, level by level,
//     r = b - A S b,   b_c = Pt^T b,   z = S (b + r) + Pt x_c,   Pt = (I - S A) P,
// because P^T (I - A S) = ((I - S A) P)^T for a symmetric A. Per level this is two dependent
// products on the cycle's critical path (the restriction by Pt^T and the prolongation by Pt)
// instead of four, and the residual, which only the prolongation of the same level reads, runs on
// a second stream beside the coarser levels.
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
    int lpr = 1;    // threads per row in the row-block kernel's sums (1, or 8 for long rows)
    const int2* rb = nullptr;
    int* err = nullptr;  // set to 1 when a staged copy never lands (never in a correct run)
    const int* ptr = nullptr;
    const int* col = nullptr;
    const T* val = nullptr;
    int nwb = 0;                // warp blocks: block w covers rows [wb[w].x, wb[w + 1].x), entries [wb[w].y, wb[w + 1].y)
    const int2* wb = nullptr;
};

// coarsest level: at most this many rows, inverted densely (2500^2 doubles = 50 MB)
constexpr int COARSE_MAX = 2500;
// largest coarsest level accepted when coarsening stops early (level cap)
constexpr int DENSE_MAX = 4096;

class Amg {
public:
    Amg() = default;
    Amg(const Amg&) = delete;
    Amg& operator=(const Amg&) = delete;
    ~Amg();
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
        int lpr = 1;          // threads per row of the row-block sums
        std::vector<int> rb;  // row blocks: (first row, first entry) pairs, one past the last block included
        std::vector<int> wb;  // warp blocks (at most 32 rows and WS_CAP entries), same layout
        std::vector<double> cval;
    };
    struct CsrBufs {  // one CSR matrix on the device: row blocks, pattern, FP64 and FP32 values
        DevBuf<int> ptr, col, rb, wb;
        DevBuf<double> v64;
        DevBuf<float> v32;
    };
    struct Level {
        int n = 0, nc = 0;
        double omega = 0;
        // A: the level's operator with its columns scaled by S = omega D^{-1} (A S, for the residual
        // r = b - A S b); Pt = (I - S A) P: n x nc, Rt = Pt^T: nc x n (absent on the coarsest level)
        Sell A, Pt, Rt;
        std::vector<double> dinv;
        // structure kept for refresh(): stored CSR pattern of A, aggregate of every stored row (empty
        // when the prolongator is given), position in P of every R entry and in Pt of every Rt entry,
        // SELL slot of every CSR entry of A (SELL storage), patterns of P and R = P^T (FP64 values:
        // the Galerkin product of the next level is R A P)
        std::vector<int> pa_ptr, pa_col, agg, r2p, rt2pt;
        std::vector<long long> sellpos;
        bool fixedP = false;
        DevBuf<int> dpa_ptr, dpa_col, dagg, dr2p, drt2pt;
        DevBuf<long long> dsellpos;
        DevBuf<double> dvals;  // unscaled stored values of A (levels below the finest; refresh)
        CsrBufs cP, cR;        // P and R (FP64 values only; refresh)
        // device storage of the cycle's matrices
        DevBuf<long long> dA_soff;
        DevBuf<int> dA_w, dA_col;
        DevBuf<double> dA_v64;
        DevBuf<float> dA_v32;
        CsrBufs cA, cPt, cRt;
        DevBuf<double> dinv64, x64, b64, r64;
        DevBuf<float> dinv32, x32, b32, r32;
    };
    template <typename T>
    void cycle(int l, const T* b, T* z, cudaStream_t s);
    void dense_inverse_device(const std::vector<double>& a, int n);
    void dense_inverse_of(double* d, int n);  // in-place device matrix -> dinvc64_ / dinvc32_
    template <typename T>
    DevSell<T> view(const Level& L) const;
    template <typename T>
    DevCsr<T> cview(const Sell& S, const CsrBufs& B) const;

    std::vector<Level> levels_;
    int ncoarse_ = 0;
    DevBuf<int> err_;
    int csr_slots_[2] = {1, 1};  // resident CTAs of the CSR kernels on this hierarchy's device (FP32, FP64)
    DevBuf<double> dinvc64_;  // dense inverse of the coarsest matrix
    DevBuf<float> dinvc32_;
    // second stream of the cycle (the residuals) and, per level, the events that fork it after the
    // level's right-hand side is written and join it before the level's prolongation
    cudaStream_t side_ = nullptr;
    std::vector<cudaEvent_t> ev_fork_, ev_join_;
    void release_streams();
};

}  // namespace vg
