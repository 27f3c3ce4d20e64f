// Learned factorised sparse approximate inverse (FSAI) preconditioner.
//
// A per-edge MLP (16 -> 64 -> 64 -> 64 -> 1, tanh-form GELU; bf16 tensor-core
// operands, fp32 accumulation) reads local matrix entries and particle
// geometry and emits G on the lower pattern of A.  M = G^T G is SPD for any
// output (G lower triangular with a positive diagonal).  G is kept aligned
// with A's CSR entries,
//
//   g[k] for the entry k = (i, j) of A:  j <= i: G_ij;  j > i: G_ji
//
// (row i's lower half holds row i of G, its upper half row i of G^T), and the
// solver applies z = G^T (G r) from compact FP16 copies of the two halves.
//
// The network is trained on the GPU by the kernels of fsai.cu: forward and
// backward of the MLP on the tensor cores (mma.sync m16n8k16 bf16), the loss
// ||G A G^T z - z||^2 over 16 Rademacher probes with its gradient dL/dG
// through probe-block SpMMs, and Adam.  The reference has no counterpart.
#pragma once

#include "common.cuh"
#include "numerics.cuh"
#include "scan.cuh"

namespace sb {

constexpr int kFsaiNF = 16;   // input features (10 used, 11 by KY-based models; zero padded to one k16 step)
constexpr int kFsaiHid = 64;  // hidden width
constexpr int kFsaiProbes = 16;
// Parameter vector (fp32 master copy): W1[16][64] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] w4[64] b4 — matrices row-major, input index first.
constexpr uint32_t kOffW1 = 0, kOffB1 = 1024, kOffW2 = 1088, kOffB2 = 5184, kOffW3 = 5248, kOffB3 = 9344,
                   kOffW4 = 9408, kOffB4 = 9472, kFsaiParamCount = 9473;
// bf16 B-operand fragments (uint2 per lane per (k-tile, n-tile)): W1, W2, W3, W2^T, W3^T.
constexpr uint32_t kFragW1 = 0, kFragW2 = 8 * 32, kFragW3 = kFragW2 + 32 * 32, kFragW2T = kFragW3 + 32 * 32,
                   kFragW3T = kFragW2T + 32 * 32, kFragCount = kFragW3T + 32 * 32;
constexpr float kFsaiDiagClip = 4.0f;
// Training losses over the probe block Z (n x 16):
//   residual: sum_p ||G A G^T z_p - z_p||^2 / (16 n);
//   kaporin:  log(t / n) - (2/n) sum_i log G_ii, t = sum_p z_p^T G A G^T z_p / 16
//             (the log of Kaporin's condition number of G A G^T up to log(det A)/n,
//             the functional the Kolotilina-Yeremin FSAI minimises).
constexpr uint32_t kFsaiLossResidual = 0, kFsaiLossKaporin = 1;
// What the network's output corrects: none (G_ij = out / sqrt(d_j), G_ii =
// exp(out) / sqrt(d_i); zero output = Jacobi), or the Kolotilina-Yeremin G
// K of the system (G_ij = K_ij + out / sqrt(d_j), G_ii = exp(out) K_ii; zero
// output = K; K_ij sqrt(d_j) is input feature 10).
constexpr uint32_t kFsaiBaseNone = 0, kFsaiBaseKy = 1;

struct FsaiModel {
    DeviceBuffer<float> params, grad, m, v;  // master weights, gradient, Adam moments
    DeviceBuffer<float> gsum;                // gradient accumulated over a batch of systems
    DeviceBuffer<uint2> frags;               // packed bf16 fragments of the current params
    DeviceBuffer<float> partials;            // per-block gradient partials
    DeviceBuffer<double> acc;                // loss accumulator
    uint32_t adam_t = 0;
    uint32_t loss_kind = 0;                  // kFsaiLossResidual or kFsaiLossKaporin
    uint32_t base = 0;                       // kFsaiBaseNone or kFsaiBaseKy
    uint64_t version = 1;                    // bumped whenever params change
    bool packed = false;
    FsaiModel();
    void pack(cudaStream_t s);
};

// Per-system data of the preconditioner (depends on A and the coordinates;
// g also on the model).
struct FsaiSystem {
    uint32_t n = 0, nnz = 0, n_edges = 0, n_upper = 0;  // n_edges: lower entries; n_upper: upper entries
    bool prepared = false;
    uint64_t g_version = 0;                   // model version g was computed with
    const FsaiModel* g_model = nullptr;
    DeviceBuffer<uint32_t> dpos, lcnt, loff;  // diagonal position, lower counts and offsets per row
    DeviceBuffer<uint32_t> e_row, e_pos;      // lower edges: row and position in A
    DeviceBuffer<float4> node;                // {log d - lmean, 1/sqrt(d), bnd, free}
    DeviceBuffer<double> red;                 // sum log d (free rows), free rows, sum dist, lower pairs
    DeviceBuffer<float> g;                    // G values aligned with A's entries
    // The solver's copies of G: compact CSR of the lower half (row offsets
    // loff, columns lcol) and of the upper half (uoff, ucol) with FP16 values
    // scaled by 2^(8 - ceil(log2 max|G|)).
    DeviceBuffer<uint32_t> lcol, ucnt, uoff, ucol;
    DeviceBuffer<__half> lval, uval;
    DeviceBuffer<float> gmax;
    DeviceBuffer<float> dG;                   // dL/dG per lower edge (training)
    DeviceBuffer<float> Z, Y, W, E, T;        // n x 16 probe blocks (training)
    DeviceBuffer<uint32_t> words;             // [0] error bits: 1 missing/non-positive diagonal, 2 unsymmetric pattern
    ScanPlan scan;
    float inv_h = 1.f;
    double setup_ms = 0, infer_ms = 0;
    uint32_t error = 0;
    bool g_ky = false;                        // g holds the Kolotilina-Yeremin G (fsai_ky)
    uint32_t ky_diag_rows = 0;                // rows the KY pass left diagonal (too long, or not positive in float)
    DeviceBuffer<float> ky;                   // the KY G aligned with A's entries (base of KY-based models)
    bool ky_ready = false;
    void invalidate() { prepared = false; g_model = nullptr; g_version = 0; g_ky = false; ky_ready = false; }
};

// Node data, lower edges and feature scalars of A (xyz: float4 per node or null).
void fsai_prepare(const CsrF64& A, const float4* xyz, FsaiSystem& S, cudaStream_t s);
// Evaluate the network on every lower edge and fill S.g (both halves).
void fsai_infer(FsaiModel& M, const CsrF64& A, const float4* xyz, FsaiSystem& S, cudaStream_t s);
// The Kolotilina-Yeremin FSAI on A's lower pattern (exact local solves, no
// model) into S.g, same layout and solver copies as fsai_infer.
void fsai_ky(const CsrF64& A, const float4* xyz, FsaiSystem& S, cudaStream_t s);
// Features of the lower edges as fp32 (n_edges x 16), for checks.
void fsai_features(const CsrF64& A, const float4* xyz, FsaiSystem& S, float* out, cudaStream_t s,
                   bool ky = false);
// Loss M.loss_kind over 16 probes (from seed, or z_host n x 16 when non-null)
// and its gradient into M.grad.  Returns the loss.
double fsai_loss_grad(FsaiModel& M, const CsrF64& A, const float4* xyz, FsaiSystem& S, uint64_t seed,
                      const float* z_host, cudaStream_t s);
// Adam step on M.params from M.grad (gradient clipped to global norm clip if clip > 0).
void fsai_adam(FsaiModel& M, float lr, float clip, cudaStream_t s);
// gsum = (first ? 0 : gsum) + w * grad; with last, grad = gsum afterwards.
void fsai_accumulate(FsaiModel& M, float w, bool first, bool last, cudaStream_t s);

}  // namespace sb
