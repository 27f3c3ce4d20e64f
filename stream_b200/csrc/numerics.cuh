// Sparse linear algebra of the pressure solve on B200.
//
// * CsrF32 / FP32 CG and Jacobi-PCG with the reference's recurrence and
//   stopping rule (src/numerics/conjugate_gradient.cpp:61-208,
//   src/numerics/preconditioner_jacobi.cpp:33-60): sqrt(r.z) <= 1e-6 absolute,
//   at most 10000 counted iterations.
// * CsrF64 / FP64 Jacobi-PCG with a relative stop ||r|| <= tol ||b||.
// * Mixed precision: FP32 matrix values, vectors and preconditioner (int32
//   indices) inside an FP64 iterative-refinement loop; residual r = b - Ax,
//   the alpha/beta dot products and the convergence check stay FP64.
// * P1 Laplacian assembly on the alpha-shape tets with Dirichlet rows.
//
// Device-side CG: every scalar (alpha, beta, dots, iteration counter, done
// flag) lives in device memory, so iterations are enqueued without host
// round trips; the host polls the done flag every kPollEvery iterations.
#pragma once

#include <cuda_fp16.h>

#include "common.cuh"
#include "scan.cuh"

namespace sb {

struct CsrF32 {
    uint32_t n = 0, nnz = 0;
    DeviceBuffer<uint32_t> row, col;
    DeviceBuffer<float> val;
};

// Largest |v| over m values into *out (device).
void absmax_f32(const float* v, uint32_t m, float* out, cudaStream_t s);

struct CsrF64 {
    uint32_t n = 0, nnz = 0;
    DeviceBuffer<uint32_t> row, col;
    DeviceBuffer<double> val;
    DeviceBuffer<float> val32;  // FP32 copy for the mixed-precision inner solver
    bool val32_ready = false;   // val32 holds the current values (the buffer is kept across changes)
    void make_f32(cudaStream_t s);
    // Derived copies are rebuilt after the matrix changes.
    void invalidate_derived() { val32_ready = false; }
};

// Device scalars of one CG run (double-buffered accumulators by iteration
// parity).  The iteration state lives here, not in kernel arguments, so that
// a captured batch of iterations can be replayed.
struct CgScalars {
    double dq[2];      // d . Ad
    double rz[2];      // r . z (z = M^-1 r)
    double rr[2];      // r . r
    double bnorm2;
    double tol2;       // relative stop: r.r <= tol2 * b.b
    uint32_t it;       // iteration counter (reference semantics for the FP32 solver)
    uint32_t done;     // 1 converged, 2 iteration cap, 3 non-finite breakdown
    uint32_t kbase;    // first iteration of the batch being replayed
    uint32_t maxit;    // bodies
};

struct CgWork {
    DeviceBuffer<CgScalars> sc;
    DeviceBuffer<double> r, z, d, q;    // FP64 vectors
    DeviceBuffer<float> r32, z32, d32, q32, x32, idiag32, y32;
    DeviceBuffer<double> idiag;
    DeviceBuffer<double> acc;           // residual-norm accumulators
    PinnedWords pinned;
};

struct SolveReport {
    uint32_t iterations = 0;        // total CG bodies (inner ones for mixed)
    uint32_t outer = 0;             // refinement steps (mixed)
    double relres = 0.0;            // true ||b - Ax|| / ||b|| in FP64, recomputed after the solve
    double ms = 0.0;                // device time of the solve
    uint32_t converged = 0;
    uint32_t fallback = 0;          // 1: the learned preconditioner stagnated and Jacobi-PCG finished the solve
};

// Learned FSAI factor G as two compact CSR matrices with scaled FP16 values:
// lower (row i of G) and upper (row i of G^T); z = G^T (G r) up to a constant
// factor (which does not change the preconditioned CG iterates).
struct FsaiOperator {
    const uint32_t* lrow = nullptr;
    const uint32_t* lcol = nullptr;
    const __half* lval = nullptr;
    const uint32_t* urow = nullptr;
    const uint32_t* ucol = nullptr;
    const __half* uval = nullptr;
};

constexpr int kPollEvery = 16;     // iterations per captured batch (even: parity slots)
// Segment target of the mixed-precision solvers: an FP32 segment runs until
// its residual has dropped 100x, then the true FP64 residual replaces it and
// the iteration continues with its search direction (measured best of
// 1e-1..3e-5 over the 1M and 4M dam-break systems; 1e-3 and below let the FP32
// drift grow and cost iterations).
constexpr double kMixedSegment = 1e-2;

// Reference FP32 solvers.  x (device, n) is in/out.  Returns the reference's
// iteration counter.
// done (may be null) receives the termination: 1 the reference's stopping
// rule, 2 its 10,000-iteration cap, 3 a non-finite r.z (breakdown).
uint32_t cg_f32_reference(const CsrF32& A, const float* b, float* x, bool jacobi, CgWork& w, cudaStream_t s,
                          uint32_t* done = nullptr);
// Number of rows whose diagonal entry is missing, zero, or has no finite inverse.
uint32_t count_bad_diagonal(const CsrF32& A, CgWork& w, cudaStream_t s);

// FP64 Jacobi-PCG to ||r|| <= rtol ||b||.  x (device) in/out.
SolveReport pcg_f64(const CsrF64& A, const double* b, double* x, double rtol, uint32_t maxit, CgWork& w,
                    cudaStream_t s);

// Mixed-precision Jacobi-PCG: FP32 iterations in segments that each reduce
// the residual by inner_rtol (<= 0: max(kMixedSegment, 0.5 rtol ||b|| /
// ||r||), so that the last one stops where the tolerance is met); after each,
// the correction is added to the FP64 x and the FP64 residual b - Ax replaces
// the FP32 one, the search direction being kept (reliable updates).  x
// (device, FP64) in/out.
SolveReport ir_mixed(const CsrF64& A, const double* b, double* x, double rtol, uint32_t maxit, double inner_rtol,
                     CgWork& w, cudaStream_t s);

// Mixed-precision PCG with the learned FSAI preconditioner: FP32 iterations
// with z = G^T (G r) in segments; after each segment (residual reduced by
// inner_rtol, or with inner_rtol <= 0 by max(kMixedSegment, 0.5 rtol ||b|| /
// ||r||)) the correction is added to the FP64 x, the FP64 residual b - Ax
// replaces the FP32 one and the iteration goes on with its search direction
// (reliable updates).  When a segment fails to halve the true residual (or
// produces a non-finite one), the solve falls back to FP64 Jacobi-PCG from the
// current iterate, or from 0 if that is better (report.fallback = 1).
SolveReport ir_fsai(const CsrF64& A, const double* b, double* x, double rtol, uint32_t maxit, double inner_rtol,
                    const FsaiOperator& G, CgWork& w, cudaStream_t s);

// True relative residual ||b - Ax|| / ||b|| in FP64 (device computation).
double relres_f64(const CsrF64& A, const double* b, const double* x, CgWork& w, cudaStream_t s);

// ---- P1 assembly ---------------------------------------------------------------
struct DivModes {  // RHS = div u, u = sum_m a_m sin(k_m . x + phi_m)
    int count = 0;
    float k[8][3];
    float adotk[8];
    float phi[8];
};

struct Assembly {
    DeviceBuffer<uint32_t> deg, off, cur, inc, cnt;
    DeviceBuffer<uint32_t> words;  // overflow and isolated-node counters
    DeviceBuffer<uint32_t> tmp;    // row columns in bounded slots (1 + 3 x incident elements per node)
    DeviceBuffer<uint32_t> incpos; // per incident element: row positions of its 4 vertices (bytes)
    ScanPlan scan;
    uint32_t n_isolated = 0, overflow = 0;
};

// Laplacian of the P1 elements `elems` (n_elems x {a,b,c,d}, ids < n) over
// points cm (float4 x,y,z,_).  Rows of nodes with is_bnd != 0 (and of nodes
// without incident element) become identity rows with zero RHS; their columns
// are eliminated from the other rows.  rhs_kind 0: f = 1; 1: f = div u (modes).
void assemble_p1_laplacian(uint32_t n, const float4* cm, const uint4* elems, uint32_t n_elems, const uint8_t* is_bnd,
                           int rhs_kind, const DivModes& modes, CsrF64& A, DeviceBuffer<double>& b, Assembly& asmb,
                           cudaStream_t s);

}  // namespace sb
