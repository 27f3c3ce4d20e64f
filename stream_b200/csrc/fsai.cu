// Learned FSAI on sm_100a: per-edge features, the MLP forward and backward on
// the tensor cores (mma.sync m16n8k16, bf16 operands, fp32 accumulators
// chained through registers from layer to layer), the probe loss and its
// gradient, Adam.  The layout of G is described in fsai.cuh.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "fsai.cuh"

namespace sb {
namespace {

constexpr int kThreads = 256;
constexpr int kMlpThreads = 128;  // 4 warps
constexpr int kXPitch = 24;       // bf16 per feature row in shared memory (conflict-free fragment loads)
constexpr int kHPitch = 72;       // bf16 per hidden row
constexpr int kTrainEdges = 64;   // edges per block step of the training kernel (16 per warp)

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    return t;  // valid in thread 0
}

// ---- tensor-core and activation helpers ------------------------------------------
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint2 b) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

__device__ __forceinline__ void ldsm_x4_trans(uint32_t (&r)[4], const void* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
    const __half2 v = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float2 unpack_h2(uint32_t u) {
    return __half22float2(*reinterpret_cast<const __half2*>(&u));
}
__device__ __forceinline__ float round_bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), and its derivative.
constexpr float kGeluC0 = 0.7978845608028654f;
constexpr float kGeluC1 = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
    const float t = tanh_fast(z * fmaf(kGeluC0 * kGeluC1, z * z, kGeluC0));
    const float h = 0.5f * z;
    return fmaf(h, t, h);
}
__device__ __forceinline__ float gelu_d(float z, float& dz) {
    const float z2 = z * z;
    const float t = tanh_fast(kGeluC0 * z * (1.0f + kGeluC1 * z2));
    dz = 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC0 * (1.0f + 3.0f * kGeluC1 * z2);
    return 0.5f * z * (1.0f + t);
}

// ---- per-edge features -----------------------------------------------------------
struct EdgeInfo {
    uint32_t pos;   // position of the entry in A
    float scale;    // dG/d(out) factor 1/sqrt(d)
    uint32_t kind;  // 0 free off-diagonal, 1 free diagonal, 2 fixed value
    float fixed;
};

struct FeatCtx {
    const uint32_t* e_row;
    const uint32_t* e_pos;
    const uint32_t* col;
    const double* val;
    const float4* node;
    const float4* xyz;
    float inv_h;
    uint32_t n_edges;
    const float* ky;  // Kolotilina-Yeremin G aligned with A's entries (KY-based models), else null
};

// Features of lower edge e: a_ij / sqrt(d_i d_j), log d_i - lmean, log d_j -
// lmean, (x_j - x_i) / h, |x_j - x_i| / h, bnd_i, bnd_j, [i == j].
__device__ __forceinline__ void edge_features(const FeatCtx& c, uint32_t e, float (&f)[kFsaiNF], EdgeInfo& info) {
    const uint32_t i = c.e_row[e], k = c.e_pos[e], j = c.col[k];
    const double av = c.val[k];
    const float a = (float)av;
    const float4 ni = c.node[i], nj = c.node[j];
#pragma unroll
    for (int t = 0; t < kFsaiNF; ++t) f[t] = 0.f;
    f[0] = a * ni.y * nj.y;
    f[1] = ni.x;
    f[2] = nj.x;
    if (c.xyz) {
        const float4 xi = c.xyz[i], xj = c.xyz[j];
        const float dx = (xj.x - xi.x) * c.inv_h, dy = (xj.y - xi.y) * c.inv_h, dz = (xj.z - xi.z) * c.inv_h;
        f[3] = dx;
        f[4] = dy;
        f[5] = dz;
        f[6] = sqrtf(dx * dx + dy * dy + dz * dz);
    }
    f[7] = ni.z;
    f[8] = nj.z;
    f[9] = i == j ? 1.f : 0.f;
    const float ky = c.ky ? c.ky[k] : 0.f;
    if (c.ky) f[10] = ky / nj.y;  // the Kolotilina-Yeremin G_ij in output units (x sqrt(d_j))
    info.pos = k;
    info.scale = 0.f;
    info.fixed = 0.f;
    if (ni.w == 0.f) {
        info.kind = 2;
        info.fixed = i == j ? ni.y : 0.f;
    } else if (i == j) {
        info.kind = 1;
        info.scale = c.ky ? ky : ni.y;  // G_ii = exp(out) x (KY G_ii or 1/sqrt(d_i))
    } else if (av == 0.0) {
        info.kind = 2;
    } else {
        info.kind = 0;
        info.scale = nj.y;
        info.fixed = ky;  // G_ij = KY G_ij + out / sqrt(d_j)  (0 without a base)
    }
}

// Lane l < 16 writes the bf16 feature row of edge base + l (zeros past the end).
__device__ __forceinline__ void stage_features(const FeatCtx& c, uint32_t e, __nv_bfloat16* xrow, EdgeInfo& info) {
    float f[kFsaiNF];
    if (e < c.n_edges) {
        edge_features(c, e, f, info);
    } else {
#pragma unroll
        for (int t = 0; t < kFsaiNF; ++t) f[t] = 0.f;
        info = EdgeInfo{0u, 0.f, 3u, 0.f};  // kind 3: padding, never written
    }
    uint32_t w[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) w[t] = pack_bf16(f[2 * t], f[2 * t + 1]);
    uint4* dst = reinterpret_cast<uint4*>(xrow);
    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

__device__ __forceinline__ float g_value(const EdgeInfo& info, float out) {
    if (info.kind == 0) return info.fixed != 0.f ? info.fixed + out * info.scale : out * info.scale;
    if (info.kind == 1) return expf(fminf(fmaxf(out, -kFsaiDiagClip), kFsaiDiagClip)) * info.scale;
    return info.fixed;
}
__device__ __forceinline__ float g_deriv(const EdgeInfo& info, float out) {
    if (info.kind == 0) return info.scale;
    if (info.kind == 1) return fabsf(out) < kFsaiDiagClip ? expf(out) * info.scale : 0.f;
    return 0.f;
}

// ---- MLP forward of one 16-edge tile (one warp) -------------------------------------
struct MlpConsts {
    const uint2* frag;  // shared
    const float* b1;
    const float* b2;
    const float* b3;
    const float* w4;    // bf16-rounded
    float b4;
};

// GELU of the accumulators of one layer, packed into the A fragments of the
// next layer (n-tiles 2kt, 2kt+1 -> k-tile kt).  kTrain also stores the bf16
// activations to H and the derivatives (half2) to DG, the slot that the
// layer's input gradient later overwrites (the same lane owns both).
template <bool kTrain>
__device__ __forceinline__ void activate(const float (&c)[8][4], uint32_t (&a)[4][4], __nv_bfloat16* H,
                                         __nv_bfloat16* DG, int g, int q) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        float h0, h1, h2, h3;
        if (kTrain) {
            float d0, d1, d2, d3;
            h0 = gelu_d(c[nt][0], d0);
            h1 = gelu_d(c[nt][1], d1);
            h2 = gelu_d(c[nt][2], d2);
            h3 = gelu_d(c[nt][3], d3);
            *reinterpret_cast<uint32_t*>(&DG[g * kHPitch + 8 * nt + 2 * q]) = pack_h2(d0, d1);
            *reinterpret_cast<uint32_t*>(&DG[(g + 8) * kHPitch + 8 * nt + 2 * q]) = pack_h2(d2, d3);
        } else {
            h0 = gelu(c[nt][0]);
            h1 = gelu(c[nt][1]);
            h2 = gelu(c[nt][2]);
            h3 = gelu(c[nt][3]);
        }
        const uint32_t lo = pack_bf16(h0, h1), hi = pack_bf16(h2, h3);
        a[nt >> 1][2 * (nt & 1)] = lo;
        a[nt >> 1][2 * (nt & 1) + 1] = hi;
        if (kTrain) {
            *reinterpret_cast<uint32_t*>(&H[g * kHPitch + 8 * nt + 2 * q]) = lo;
            *reinterpret_cast<uint32_t*>(&H[(g + 8) * kHPitch + 8 * nt + 2 * q]) = hi;
        }
    }
}

__device__ __forceinline__ void bias_init(float (&c)[8][4], const float* b, int q) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float2 bb = *reinterpret_cast<const float2*>(&b[8 * nt + 2 * q]);
        c[nt][0] = bb.x;
        c[nt][1] = bb.y;
        c[nt][2] = bb.x;
        c[nt][3] = bb.y;
    }
}

__device__ __forceinline__ void hidden_layer(float (&c)[8][4], const uint32_t (&a)[4][4], const uint2* frag, int lane) {
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) mma_bf16(c[nt], a[kt], frag[(kt * 8 + nt) * 32 + lane]);
}

// Output of rows g and g+8 of the tile (identical in the 4 lanes of a quad).
template <bool kTrain>
__device__ __forceinline__ void mlp_forward(const MlpConsts& W, const __nv_bfloat16* X, int lane, float (&out)[2],
                                            __nv_bfloat16* H1, __nv_bfloat16* H2, float* H3, __nv_bfloat16* DG1,
                                            __nv_bfloat16* DG2, uint32_t (&dg3)[16]) {
    const int g = lane >> 2, q = lane & 3;
    uint32_t xa[4];
    xa[0] = *reinterpret_cast<const uint32_t*>(&X[g * kXPitch + 2 * q]);
    xa[1] = *reinterpret_cast<const uint32_t*>(&X[(g + 8) * kXPitch + 2 * q]);
    xa[2] = *reinterpret_cast<const uint32_t*>(&X[g * kXPitch + 2 * q + 8]);
    xa[3] = *reinterpret_cast<const uint32_t*>(&X[(g + 8) * kXPitch + 2 * q + 8]);
    float c[8][4];
    bias_init(c, W.b1, q);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) mma_bf16(c[nt], xa, W.frag[kFragW1 + nt * 32 + lane]);
    uint32_t a[4][4];
    activate<kTrain>(c, a, H1, DG1, g, q);
    bias_init(c, W.b2, q);
    hidden_layer(c, a, W.frag + kFragW2, lane);
    activate<kTrain>(c, a, H2, DG2, g, q);
    bias_init(c, W.b3, q);
    hidden_layer(c, a, W.frag + kFragW3, lane);
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float2 w = *reinterpret_cast<const float2*>(&W.w4[8 * nt + 2 * q]);
        float h[4];
        if (kTrain) {
            float d[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) h[r] = gelu_d(c[nt][r], d[r]);
            dg3[2 * nt] = pack_h2(d[0], d[1]);
            dg3[2 * nt + 1] = pack_h2(d[2], d[3]);
            *reinterpret_cast<float2*>(&H3[g * kFsaiHid + 8 * nt + 2 * q]) = make_float2(h[0], h[1]);
            *reinterpret_cast<float2*>(&H3[(g + 8) * kFsaiHid + 8 * nt + 2 * q]) = make_float2(h[2], h[3]);
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r) h[r] = gelu(c[nt][r]);
        }
        s0 += h[0] * w.x + h[1] * w.y;
        s1 += h[2] * w.x + h[3] * w.y;
    }
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    out[0] = s0 + W.b4;
    out[1] = s1 + W.b4;
}

// Shared-memory copies of the packed weights and the fp32 vectors.
__device__ __forceinline__ void load_weights(const float* __restrict__ P, const uint2* __restrict__ frags, uint2* sfrag,
                                             uint32_t nfrag, float* sb1, float* sb2, float* sb3, float* sw4,
                                             float* sb4) {
    for (uint32_t t = threadIdx.x; t < nfrag; t += blockDim.x) sfrag[t] = frags[t];
    for (uint32_t t = threadIdx.x; t < (uint32_t)kFsaiHid; t += blockDim.x) {
        sb1[t] = P[kOffB1 + t];
        sb2[t] = P[kOffB2 + t];
        sb3[t] = P[kOffB3 + t];
        sw4[t] = round_bf16(P[kOffW4 + t]);
    }
    if (threadIdx.x == 0) *sb4 = P[kOffB4];
    __syncthreads();
}

// ---- training: forward + backward, per-block gradient partials ------------------------
struct TrainSmem {
    uint2 frag[kFragCount];
    float b1[kFsaiHid], b2[kFsaiHid], b3[kFsaiHid], w4[kFsaiHid];
    float b4;
    __align__(16) __nv_bfloat16 X[kTrainEdges * kXPitch];
    __align__(16) __nv_bfloat16 H1[kTrainEdges * kHPitch];
    __align__(16) __nv_bfloat16 H2[kTrainEdges * kHPitch];
    __align__(16) __nv_bfloat16 D1[kTrainEdges * kHPitch];
    __align__(16) __nv_bfloat16 D2[kTrainEdges * kHPitch];
    __align__(16) __nv_bfloat16 D3[kTrainEdges * kHPitch];
    __align__(16) float H3[kTrainEdges * kFsaiHid];
    float dout[kTrainEdges];
    float dgv[kTrainEdges];
    EdgeInfo info[kTrainEdges];
};

// dz = (accumulator) * gelu'(z), packed to bf16 A fragments and stored to D.
// The derivatives come from registers (dg) or, when dg is null, from D itself.
__device__ __forceinline__ void grad_to_frags(const float (&c)[8][4], const uint32_t* dg, uint32_t (&a)[4][4],
                                              __nv_bfloat16* D, int g, int q) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        uint32_t* lo_p = reinterpret_cast<uint32_t*>(&D[g * kHPitch + 8 * nt + 2 * q]);
        uint32_t* hi_p = reinterpret_cast<uint32_t*>(&D[(g + 8) * kHPitch + 8 * nt + 2 * q]);
        const float2 d01 = unpack_h2(dg ? dg[2 * nt] : *lo_p), d23 = unpack_h2(dg ? dg[2 * nt + 1] : *hi_p);
        const uint32_t lo = pack_bf16(c[nt][0] * d01.x, c[nt][1] * d01.y);
        const uint32_t hi = pack_bf16(c[nt][2] * d23.x, c[nt][3] * d23.y);
        a[nt >> 1][2 * (nt & 1)] = lo;
        a[nt >> 1][2 * (nt & 1) + 1] = hi;
        *lo_p = lo;
        *hi_p = hi;
    }
}

__global__ void __launch_bounds__(kMlpThreads) k_fsai_train(FeatCtx fc, const float* __restrict__ P,
                                                            const uint2* __restrict__ frags,
                                                            const float* __restrict__ dG, float* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& sm = *reinterpret_cast<TrainSmem*>(smem_raw);
    load_weights(P, frags, sm.frag, kFragCount, sm.b1, sm.b2, sm.b3, sm.w4, &sm.b4);
    const MlpConsts W{sm.frag, sm.b1, sm.b2, sm.b3, sm.w4, sm.b4};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;
    float acc1[2][4] = {}, acc2[8][4] = {}, acc3[8][4] = {};
    float pb1 = 0.f, pb2 = 0.f, pb3 = 0.f, pw4 = 0.f, pb4 = 0.f;
    const int col_t = threadIdx.x & 63, half_t = threadIdx.x >> 6;
    // ldmatrix lane addressing (see the fragment layouts of mma.m16n8k16)
    const int lm_row_a = ((lane >> 4) & 1) * 8 + (lane & 7), lm_col_a = ((lane >> 3) & 1) * 8;
    const int lm_row_b = ((lane >> 3) & 1) * 8 + (lane & 7), lm_col_b = ((lane >> 4) & 1) * 8;

    for (uint32_t base = blockIdx.x * kTrainEdges; base < fc.n_edges; base += gridDim.x * kTrainEdges) {
        const int r0 = 16 * w;  // this warp's rows in the block tile
        if (lane < 16) {
            const uint32_t e = base + r0 + lane;
            stage_features(fc, e, &sm.X[(r0 + lane) * kXPitch], sm.info[r0 + lane]);
            sm.dgv[r0 + lane] = e < fc.n_edges ? dG[e] : 0.f;
        }
        __syncwarp();
        uint32_t dg3[16];
        float out[2];
        mlp_forward<true>(W, &sm.X[r0 * kXPitch], lane, out, &sm.H1[r0 * kHPitch], &sm.H2[r0 * kHPitch],
                          &sm.H3[r0 * kFsaiHid], &sm.D1[r0 * kHPitch], &sm.D2[r0 * kHPitch], dg3);
        float dout[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const EdgeInfo inf = sm.info[r0 + g + 8 * h];
            dout[h] = sm.dgv[r0 + g + 8 * h] * g_deriv(inf, out[h]);
        }
        if (q == 0) {
            sm.dout[r0 + g] = dout[0];
            sm.dout[r0 + g + 8] = dout[1];
        }
        // dz3 = dout w4 gelu'(z3)
        float c[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const float2 wv = *reinterpret_cast<const float2*>(&W.w4[8 * nt + 2 * q]);
            c[nt][0] = dout[0] * wv.x;
            c[nt][1] = dout[0] * wv.y;
            c[nt][2] = dout[1] * wv.x;
            c[nt][3] = dout[1] * wv.y;
        }
        uint32_t a[4][4];
        grad_to_frags(c, dg3, a, &sm.D3[r0 * kHPitch], g, q);
        // dz2 = (dz3 W3^T) gelu'(z2)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.f;
        hidden_layer(c, a, W.frag + kFragW3T, lane);
        grad_to_frags(c, nullptr, a, &sm.D2[r0 * kHPitch], g, q);
        // dz1 = (dz2 W2^T) gelu'(z1)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.f;
        hidden_layer(c, a, W.frag + kFragW2T, lane);
        grad_to_frags(c, nullptr, a, &sm.D1[r0 * kHPitch], g, q);
        __syncthreads();

        // Weight gradients over the block's 64 edges: dW2 = H1^T D2, dW3 = H2^T D3
        // (rows 16w..16w+15 in this warp), dW1 = X^T D1 (columns 16w..16w+15).
#pragma unroll
        for (int ks = 0; ks < kTrainEdges / 16; ++ks) {
            uint32_t ah1[4], ah2[4], ax[4];
            ldsm_x4_trans(ah1, &sm.H1[(16 * ks + lm_row_a) * kHPitch + 16 * w + lm_col_a]);
            ldsm_x4_trans(ah2, &sm.H2[(16 * ks + lm_row_a) * kHPitch + 16 * w + lm_col_a]);
            ldsm_x4_trans(ax, &sm.X[(16 * ks + lm_row_a) * kXPitch + lm_col_a]);
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                uint32_t b2[4], b3[4];
                ldsm_x4_trans(b2, &sm.D2[(16 * ks + lm_row_b) * kHPitch + 16 * p + lm_col_b]);
                ldsm_x4_trans(b3, &sm.D3[(16 * ks + lm_row_b) * kHPitch + 16 * p + lm_col_b]);
                mma_bf16(acc2[2 * p], ah1, make_uint2(b2[0], b2[1]));
                mma_bf16(acc2[2 * p + 1], ah1, make_uint2(b2[2], b2[3]));
                mma_bf16(acc3[2 * p], ah2, make_uint2(b3[0], b3[1]));
                mma_bf16(acc3[2 * p + 1], ah2, make_uint2(b3[2], b3[3]));
            }
            uint32_t b1[4];
            ldsm_x4_trans(b1, &sm.D1[(16 * ks + lm_row_b) * kHPitch + 16 * w + lm_col_b]);
            mma_bf16(acc1[0], ax, make_uint2(b1[0], b1[1]));
            mma_bf16(acc1[1], ax, make_uint2(b1[2], b1[3]));
        }
        // Bias and output-layer gradients: column sums over this thread's 32 edges.
        for (int e = 32 * half_t; e < 32 * half_t + 32; ++e) {
            pb1 += __bfloat162float(sm.D1[e * kHPitch + col_t]);
            pb2 += __bfloat162float(sm.D2[e * kHPitch + col_t]);
            pb3 += __bfloat162float(sm.D3[e * kHPitch + col_t]);
            pw4 += sm.H3[e * kFsaiHid + col_t] * sm.dout[e];
        }
        if (threadIdx.x == 0)
            for (int e = 0; e < kTrainEdges; ++e) pb4 += sm.dout[e];
        __syncthreads();
    }

    float* out = partials + (size_t)blockIdx.x * kFsaiParamCount;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int n = 8 * (2 * w + j) + 2 * q;
        out[kOffW1 + g * kFsaiHid + n] = acc1[j][0];
        out[kOffW1 + g * kFsaiHid + n + 1] = acc1[j][1];
        out[kOffW1 + (g + 8) * kFsaiHid + n] = acc1[j][2];
        out[kOffW1 + (g + 8) * kFsaiHid + n + 1] = acc1[j][3];
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int m = 16 * w + g, n = 8 * nt + 2 * q;
        out[kOffW2 + m * kFsaiHid + n] = acc2[nt][0];
        out[kOffW2 + m * kFsaiHid + n + 1] = acc2[nt][1];
        out[kOffW2 + (m + 8) * kFsaiHid + n] = acc2[nt][2];
        out[kOffW2 + (m + 8) * kFsaiHid + n + 1] = acc2[nt][3];
        out[kOffW3 + m * kFsaiHid + n] = acc3[nt][0];
        out[kOffW3 + m * kFsaiHid + n + 1] = acc3[nt][1];
        out[kOffW3 + (m + 8) * kFsaiHid + n] = acc3[nt][2];
        out[kOffW3 + (m + 8) * kFsaiHid + n + 1] = acc3[nt][3];
    }
    float* red = sm.H3;  // reuse: [4][64]
    if (half_t == 1) {
        red[col_t] = pb1;
        red[64 + col_t] = pb2;
        red[128 + col_t] = pb3;
        red[192 + col_t] = pw4;
    }
    __syncthreads();
    if (half_t == 0) {
        out[kOffB1 + col_t] = pb1 + red[col_t];
        out[kOffB2 + col_t] = pb2 + red[64 + col_t];
        out[kOffB3 + col_t] = pb3 + red[128 + col_t];
        out[kOffW4 + col_t] = pw4 + red[192 + col_t];
    }
    if (threadIdx.x == 0) out[kOffB4] = pb4;
}

__global__ void k_fsai_reduce(const float* __restrict__ partials, uint32_t nblk, float* __restrict__ grad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kFsaiParamCount) return;
    float s = 0.f;
    for (uint32_t b = 0; b < nblk; ++b) s += partials[(size_t)b * kFsaiParamCount + i];
    grad[i] = s;
}

// ---- weights -> bf16 fragments ------------------------------------------------------
__global__ void k_fsai_pack(const float* __restrict__ P, uint2* __restrict__ frag) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kFragCount) return;
    uint32_t off, f;
    bool trans;
    if (t < kFragW2) { off = kOffW1; f = t; trans = false; }
    else if (t < kFragW3) { off = kOffW2; f = t - kFragW2; trans = false; }
    else if (t < kFragW2T) { off = kOffW3; f = t - kFragW3; trans = false; }
    else if (t < kFragW3T) { off = kOffW2; f = t - kFragW2T; trans = true; }
    else { off = kOffW3; f = t - kFragW3T; trans = true; }
    const uint32_t lane = f & 31, nt = (f >> 5) & 7, kt = f >> 8;
    const uint32_t n = 8 * nt + (lane >> 2), k0 = 16 * kt + 2 * (lane & 3);
    // B[k][n] = W[k][n] (forward) or W[n][k] (backward, W^T)
    auto e = [&](uint32_t k) { return trans ? P[off + n * kFsaiHid + k] : P[off + k * kFsaiHid + n]; };
    frag[t] = make_uint2(pack_bf16(e(k0), e(k0 + 1)), pack_bf16(e(k0 + 8), e(k0 + 9)));
}

// ---- node data and lower edges --------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_fsai_rows(uint32_t n, const uint32_t* __restrict__ row,
                                                        const uint32_t* __restrict__ col, const double* __restrict__ val,
                                                        const float4* __restrict__ xyz, uint32_t* __restrict__ dpos,
                                                        uint32_t* __restrict__ lcnt, float4* __restrict__ node,
                                                        double* red, uint32_t* err) {
    __shared__ double sh[32];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double slog = 0.0, sfree = 0.0, sdist = 0.0, spair = 0.0;
    if (i < n) {
        const uint32_t r0 = row[i], r1 = row[i + 1];
        uint32_t dp = 0xffffffffu, noff = 0, nzero = 0, bad = 0;
        double d = 0.0;
        float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
        if (xyz) xi = xyz[i];
        for (uint32_t k = r0; k < r1; ++k) {
            const uint32_t j = col[k];
            const double a = val[k];
            if (k > r0 && !(col[k - 1] < j)) bad |= 4;  // strictly increasing columns
            if (j == i) {
                dp = k;
                d = a;
                continue;
            }
            if ((j < i) != (dp == 0xffffffffu)) bad |= 4;  // columns must be sorted around the diagonal
            ++noff;
            if (a == 0.0) {
                ++nzero;
            } else if (j < i && xyz) {
                const float4 xj = xyz[j];
                const double dx = (double)xj.x - xi.x, dy = (double)xj.y - xi.y, dz = (double)xj.z - xi.z;
                sdist += sqrt(dx * dx + dy * dy + dz * dz);
                spair += 1.0;
            }
        }
        if (dp == 0xffffffffu || !(d > 0.0)) bad |= 1;
        const float bnd = (noff > 0 && nzero < noff) ? (float)((double)nzero / (double)noff) : 1.f;
        const bool fr = bnd < 1.f;
        if (fr && !(bad & 1)) {
            slog = log(d);
            sfree = 1.0;
        }
        dpos[i] = bad & 1 ? r0 : dp;
        lcnt[i] = bad ? 0u : dp - r0 + 1;
        node[i] = make_float4(0.f, bad & 1 ? 0.f : (float)(1.0 / sqrt(d)), bnd, fr ? 1.f : 0.f);
        if (bad) atomicOr(err, bad);
    }
    slog = block_sum(slog, sh);
    if (threadIdx.x == 0) atomicAdd(&red[0], slog);
    sfree = block_sum(sfree, sh);
    if (threadIdx.x == 0) atomicAdd(&red[1], sfree);
    sdist = block_sum(sdist, sh);
    if (threadIdx.x == 0) atomicAdd(&red[2], sdist);
    spair = block_sum(spair, sh);
    if (threadIdx.x == 0) atomicAdd(&red[3], spair);
}

__global__ void k_fsai_nodes(uint32_t n, const uint32_t* __restrict__ dpos, const double* __restrict__ val,
                             double lmean, float4* __restrict__ node) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = val[dpos[i]];
    node[i].x = d > 0.0 ? (float)(log(d) - lmean) : 0.f;
}

__global__ void k_fsai_edges(uint32_t n, const uint32_t* __restrict__ row, const uint32_t* __restrict__ loff,
                             uint32_t* __restrict__ e_row, uint32_t* __restrict__ e_pos) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t o = loff[i], c = loff[i + 1] - o, r0 = row[i];
    for (uint32_t t = 0; t < c; ++t) {
        e_row[o + t] = i;
        e_pos[o + t] = r0 + t;
    }
}

// Upper entries take the value of their mirror: g[(i, j)] = G_ji for j > i.
__global__ void k_fsai_mirror(uint32_t n, const uint32_t* __restrict__ row, const uint32_t* __restrict__ col,
                              const uint32_t* __restrict__ dpos, float* __restrict__ g, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t k = dpos[i] + 1; k < row[i + 1]; ++k) {
        const uint32_t j = col[k];
        uint32_t lo = row[j], hi = dpos[j];
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (col[mid] < i) lo = mid + 1;
            else hi = mid;
        }
        if (lo < dpos[j] && col[lo] == i) {
            g[k] = g[lo];
        } else {
            g[k] = 0.f;
            atomicOr(err, 2u);
        }
    }
}

// Kolotilina-Yeremin FSAI on A's lower pattern (no learning): row i of G
// solves A[J,J] x = e_last, J the columns j <= i of row i (the diagonal
// last), and is scaled by 1/sqrt(x_last), so that diag(G A G^T) = 1 -- the G
// that minimises Kaporin's condition number of G A G^T over the pattern, the
// functional the learned network's Kaporin loss estimates.  One thread per
// row: the packed lower triangle of A[J,J] (float, local memory), its
// Cholesky factor in place, one back substitution.  A row longer than kKyMax
// or whose block loses positivity in float keeps the diagonal row
// 1/sqrt(a_ii) and is counted in words[1].  A register-resident variant for
// rows of up to 12 lower entries (every index fixed at compile time), with
// the longer rows in a second pass, measured slower at 1M rows (1.68 against
// 1.30 ms for the whole KY set-up).
constexpr int kKyMax = 24;
__global__ void __launch_bounds__(128) k_fsai_ky(uint32_t n, const uint32_t* __restrict__ row,
                                                 const uint32_t* __restrict__ col, const double* __restrict__ val,
                                                 const uint32_t* __restrict__ dpos, float* __restrict__ g,
                                                 uint32_t* __restrict__ words) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t b = row[i], dp = dpos[i];
    const int m = (int)(dp - b) + 1;
    float L[kKyMax * (kKyMax + 1) / 2];
    float x[kKyMax];
    bool ok = m <= kKyMax;
    if (ok) {
        for (int a = 0; a < m; ++a) {  // A[J_a][J_c], c <= a: merge row J_a with J
            const uint32_t ja = col[b + a];
            uint32_t p = row[ja];
            const uint32_t pe = row[ja + 1];
            float* La = L + a * (a + 1) / 2;
            for (int c = 0; c <= a; ++c) {
                const uint32_t jc = col[b + c];
                while (p < pe && col[p] < jc) ++p;
                La[c] = (p < pe && col[p] == jc) ? (float)val[p] : 0.f;
            }
        }
        for (int a = 0; a < m && ok; ++a) {  // A[J,J] = L L^T, row a of L
            float* La = L + a * (a + 1) / 2;
            for (int c = 0; c <= a; ++c) {
                const float* Lc = L + c * (c + 1) / 2;
                float t = La[c];
                for (int k = 0; k < c; ++k) t -= La[k] * Lc[k];
                if (c < a) La[c] = t / Lc[c];
                else if (t > 0.f) La[a] = sqrtf(t);
                else ok = false;
            }
        }
    }
    if (!ok) {
        for (uint32_t k = b; k < dp; ++k) g[k] = 0.f;
        g[dp] = (float)(1.0 / sqrt(val[dp]));
        atomicAdd(&words[1], 1u);
        return;
    }
    // L y = e_last: y = e_last / L_ll.  L^T x = y, then G's row = x * L_ll:
    // its last entry is 1 / L_ll, the others -(sum_{t>k} L_tk x_t) / L_kk.
    const float lll = L[(m - 1) * m / 2 + m - 1];
    x[m - 1] = 1.f / lll;
    for (int k = m - 2; k >= 0; --k) {
        float t = 0.f;
        for (int r = k + 1; r < m; ++r) t += L[r * (r + 1) / 2 + k] * x[r];
        x[k] = -t / L[k * (k + 1) / 2 + k];
    }
    for (int k = 0; k < m; ++k) g[b + k] = x[k];
}

__global__ void k_fsai_features(FeatCtx fc, float* __restrict__ out) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= fc.n_edges) return;
    float f[kFsaiNF];
    EdgeInfo info;
    edge_features(fc, e, f, info);
#pragma unroll
    for (int t = 0; t < kFsaiNF; ++t) out[(size_t)e * kFsaiNF + t] = f[t];
}

// ---- probe loss and dL/dG ----------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t h) {
    h ^= h >> 33;
    h *= 0xFF51AFD7ED558CCDull;
    h ^= h >> 33;
    h *= 0xC4CEB9FE1A85EC53ull;
    h ^= h >> 33;
    return h;
}

__global__ void k_fsai_probes(uint32_t n, uint64_t seed, float* __restrict__ Z) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)n * kFsaiProbes) return;
    const uint64_t h = mix64(t ^ (seed * 0x9E3779B97F4A7C15ull));
    Z[t] = (h & 1) ? 1.f : -1.f;
}

// Y = op X for a block of 16 probe columns (16 lanes per row).  kMode 0: A;
// 1: G (lower half-rows); 2: G^T (upper half-rows).  With Zsub: Y = op X - Zsub
// and the squared norm is accumulated into loss.
template <int kMode>
__global__ void __launch_bounds__(kThreads) k_fsai_spmm(uint32_t n, const uint32_t* __restrict__ row,
                                                        const uint32_t* __restrict__ col,
                                                        const uint32_t* __restrict__ dpos,
                                                        const double* __restrict__ aval, const float* __restrict__ g,
                                                        const float* __restrict__ X, float* __restrict__ Y,
                                                        const float* __restrict__ Zsub, double* loss) {
    __shared__ double sh[32];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t >> 4, p = t & 15;
    double l = 0.0;
    if (i < n) {
        uint32_t k0, k1;
        if (kMode == 0 || kMode == 3) { k0 = row[i]; k1 = row[i + 1]; }
        else if (kMode == 1) { k0 = row[i]; k1 = dpos[i] + 1; }
        else { k0 = dpos[i]; k1 = row[i + 1]; }
        float s = 0.f;
        for (uint32_t k = k0; k < k1; ++k) {
            const float v = (kMode == 0 || kMode == 3) ? (float)aval[k] : g[k];
            s += v * X[(size_t)col[k] * kFsaiProbes + p];
        }
        if (Zsub) {
            s -= Zsub[(size_t)i * kFsaiProbes + p];
            l = (double)s * s;
        }
        if (kMode == 3) l = (double)X[(size_t)i * kFsaiProbes + p] * s;  // x . (A x)
        Y[(size_t)i * kFsaiProbes + p] = s;
    }
    if (loss) {
        l = block_sum(l, sh);
        if (threadIdx.x == 0) atomicAdd(loss, l);
    }
}

// dL/dG_ij = 2/(P n) sum_p (E_ip W_jp + Z_ip T_jp) on the lower edges.
__global__ void __launch_bounds__(kThreads) k_fsai_dG(uint32_t n_edges, const uint32_t* __restrict__ e_row,
                                                      const uint32_t* __restrict__ e_pos,
                                                      const uint32_t* __restrict__ col, const float* __restrict__ E,
                                                      const float* __restrict__ W, const float* __restrict__ Z,
                                                      const float* __restrict__ T, float scale,
                                                      float* __restrict__ dG) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t e = t >> 4, p = t & 15;
    float v = 0.f;
    if (e < n_edges) {
        const size_t i = e_row[e], j = col[e_pos[e]];
        v = E[i * kFsaiProbes + p] * W[j * kFsaiProbes + p] + Z[i * kFsaiProbes + p] * T[j * kFsaiProbes + p];
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, 16);
    if (e < n_edges && p == 0) dG[e] = v * scale;
}

// Kaporin loss: dL/dG_ij = 2/ts sum_p Z_ip W_jp (ts = acc[0] = sum_p z_p^T G A G^T z_p),
// minus 2/(n G_ii) on the diagonal.
__global__ void __launch_bounds__(kThreads) k_fsai_dG_kaporin(uint32_t n, uint32_t n_edges,
                                                              const uint32_t* __restrict__ e_row,
                                                              const uint32_t* __restrict__ e_pos,
                                                              const uint32_t* __restrict__ col,
                                                              const float* __restrict__ Z, const float* __restrict__ W,
                                                              const float* __restrict__ g, const double* acc,
                                                              float* __restrict__ dG) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t e = t >> 4, p = t & 15;
    float v = 0.f;
    size_t i = 0, j = 0;
    if (e < n_edges) {
        i = e_row[e];
        j = col[e_pos[e]];
        v = Z[i * kFsaiProbes + p] * W[j * kFsaiProbes + p];
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, 16);
    if (e < n_edges && p == 0) {
        float d = (float)(2.0 / acc[0]) * v;
        if (i == j) d -= (float)(2.0 / n) / g[e_pos[e]];
        dG[e] = d;
    }
}

// acc[1] += sum_i log G_ii.
__global__ void __launch_bounds__(kThreads) k_fsai_logdiag(uint32_t n, const uint32_t* __restrict__ dpos,
                                                           const float* __restrict__ g, double* acc) {
    __shared__ double sh[32];
    double l = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        l += log((double)g[dpos[i]]);
    l = block_sum(l, sh);
    if (threadIdx.x == 0) atomicAdd(&acc[1], l);
}

// ---- Adam ------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_fsai_adam(float* __restrict__ P, const float* __restrict__ G,
                                                    float* __restrict__ m, float* __restrict__ v, float lr, float bc1,
                                                    float bc2, float clip) {
    __shared__ double sh[32];
    __shared__ float s_scale;
    double ss = 0.0;
    for (uint32_t i = threadIdx.x; i < kFsaiParamCount; i += blockDim.x) ss += (double)G[i] * G[i];
    ss = block_sum(ss, sh);
    if (threadIdx.x == 0) {
        const double nrm = sqrt(ss);
        s_scale = (clip > 0.f && nrm > clip) ? (float)(clip / nrm) : 1.f;
    }
    __syncthreads();
    const float sc = s_scale;
    constexpr float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (uint32_t i = threadIdx.x; i < kFsaiParamCount; i += blockDim.x) {
        const float gi = G[i] * sc;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        P[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

// ---- compact FP16 copies of the two halves of G (the solver's operator) ---------
__device__ __forceinline__ float half_scale(const float* gmax) {
    const float mx = *gmax;
    return mx > 0.f ? exp2f(8.f - ceilf(log2f(mx))) : 1.f;
}

__global__ void k_fsai_lower_cols(uint32_t ne, const uint32_t* __restrict__ e_pos, const uint32_t* __restrict__ col,
                                  uint32_t* __restrict__ lcol) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < ne) lcol[e] = col[e_pos[e]];
}

__global__ void k_fsai_lower_vals(uint32_t ne, const uint32_t* __restrict__ e_pos, const float* __restrict__ g,
                                  const float* __restrict__ gmax, __half* __restrict__ lval) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < ne) lval[e] = __float2half_rn(g[e_pos[e]] * half_scale(gmax));
}

__global__ void k_fsai_upper_cnt(uint32_t n, const uint32_t* __restrict__ row, const uint32_t* __restrict__ dpos,
                                 uint32_t* __restrict__ ucnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ucnt[i] = row[i + 1] - dpos[i];
}

// Row i of G^T: entries dpos[i] .. row[i+1]-1 of A's row i (columns, or
// scaled FP16 values of g).
__global__ void k_fsai_upper_fill(uint32_t n, const uint32_t* __restrict__ dpos, const uint32_t* __restrict__ uoff,
                                  const uint32_t* __restrict__ col, const float* __restrict__ g,
                                  uint32_t* __restrict__ ucol, const float* __restrict__ gmax,
                                  __half* __restrict__ uval) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t b = uoff[i], c = uoff[i + 1] - b, k0 = dpos[i];
    if (ucol) {
        for (uint32_t t = 0; t < c; ++t) ucol[b + t] = col[k0 + t];
    } else {
        const float sc = half_scale(gmax);
        for (uint32_t t = 0; t < c; ++t) uval[b + t] = __float2half_rn(g[k0 + t] * sc);
    }
}

__global__ void k_fsai_accumulate(float* __restrict__ gsum, float* __restrict__ grad, float w, int first, int last) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kFsaiParamCount) return;
    const float v = (first ? 0.f : gsum[i]) + w * grad[i];
    gsum[i] = v;
    if (last) grad[i] = v;
}

int mlp_grid(uint32_t work_items, int per_block, int cap) {
    const uint32_t b = (work_items + per_block - 1) / per_block;
    return (int)std::max<uint32_t>(1u, std::min<uint32_t>(b, (uint32_t)cap));
}

FeatCtx feat_ctx(const CsrF64& A, const float4* xyz, const FsaiSystem& S, bool ky = false) {
    return FeatCtx{S.e_row.ptr, S.e_pos.ptr, A.col.ptr, A.val.ptr, S.node.ptr, xyz, S.inv_h, S.n_edges,
                   ky ? S.ky.ptr : nullptr};
}

// ---- inference on the 5th-generation tensor cores (tcgen05) -------------------------
// A block of kTcGroups x 128 threads shares one copy of the weights; each group
// of four warps takes 128 lower edges at a time: thread r stages the features
// of edge r of the tile as row r of a 128 x 16 bf16 A tile in shared memory,
// one elected thread issues tcgen05.mma (M = 128, N = 64, bf16 x bf16 -> f32
// accumulators in tensor memory, K = 16 per instruction) against the layer's
// weights W^T (N x K, also in shared memory) and commits to the group's
// mbarrier, and each warp reads its 32 rows back with tcgen05.ld.  The
// accumulators start from the layer's bias (stored into tensor memory with
// tcgen05.st), as the training forward's mma.sync accumulators do; GELU in
// registers and the bf16 activations become the next layer's A tile.  Layer 4
// (64 -> 1) is a per-thread dot product.  The roundings are those of the
// training forward (bf16 operands and activations entering layers 2 and 3,
// f32 accumulation, f32 GELU output into layer 4).  Four groups per block and
// two blocks per SM keep 32 warps resident so that the feature gathers of one
// tile overlap the activations of the others; the kernel is bound by the
// 192 GELUs per edge (tanh on the SFU and ~6 FP32 instructions each), not by
// the 18.6 kFLOP per edge on the tensor cores.
//
// Operands use the no-swizzle K-major canonical layout: 8 x 16-byte core
// matrices (8 rows x 8 bf16) of 128 contiguous bytes; the two core matrices of
// one K = 16 step are LBO = 128 B apart and 8-row groups SBO = 128 x (K / 8)
// bytes apart.
constexpr int kTcRows = 128;
constexpr int kTcGroups = 4;                      // tiles in flight per block
constexpr int kTcBlocksPerSM = 2;
constexpr int kTcThreads = kTcRows * kTcGroups;
constexpr uint32_t kTcCols = 64;                  // tensor-memory columns per group (f32, N = 64)
constexpr uint32_t kTcAlloc = kTcCols * kTcGroups;  // a power of two in [32, 512]
static_assert(kTcBlocksPerSM * kTcAlloc <= 512, "resident blocks never wait for tensor memory");
constexpr uint32_t kTcIdesc = (1u << 4)          // D: f32
                              | (1u << 7)        // A: bf16
                              | (1u << 10)       // B: bf16 (A and B K-major, no negation)
                              | ((64u >> 3) << 17)   // N = 64
                              | ((128u >> 4) << 24); // M = 128
constexpr uint64_t kTcWaitNs = 100ull * 1000 * 1000;
constexpr uint32_t kErrTensorWait = 4u;          // words[0] bit: a tensor-core completion wait ran out

struct TcGroupSmem {
    __nv_bfloat16 A1[kTcRows * kFsaiNF];         // features: 128 x 16
    __nv_bfloat16 A2[kTcRows * kFsaiHid];        // activations: 128 x 64 (layers 2 and 3)
};

struct TcSmem {
    __nv_bfloat16 B1[kFsaiHid * kFsaiNF];        // W1^T: 64 x 16
    __nv_bfloat16 B2[kFsaiHid * kFsaiHid];       // W2^T: 64 x 64
    __nv_bfloat16 B3[kFsaiHid * kFsaiHid];       // W3^T: 64 x 64
    TcGroupSmem grp[kTcGroups];
    __align__(16) float bias[3][kFsaiHid];
    float w4[kFsaiHid];
    float b4;
    uint32_t tmem;
    uint64_t mbar[kTcGroups];
};

// Element index of (row r, k) in a K-major no-swizzle operand with kc = K / 8 chunks.
__device__ __forceinline__ uint32_t tc_idx(uint32_t r, uint32_t k, uint32_t kc) {
    return (r >> 3) * (kc * 64) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

__device__ __forceinline__ uint64_t tc_desc(const void* p, uint32_t lbo, uint32_t sbo) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

// D (+)= A B^T; accumulate = 0 overwrites D.
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(kTcIdesc), "r"(accumulate), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(bar))
                 : "memory");
}

// Wait for phase `parity` of the mbarrier; false after kTcWaitNs.
__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    uint64_t t0 = 0;
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (!t0) t0 = t;
        else if (t - t0 > kTcWaitNs) return false;
    }
}

// Barrier over the 128 threads of one group (named barrier 1 + g); returns the OR of v.
__device__ __forceinline__ bool tc_group_sync_or(uint32_t g, bool v) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(1u + g), "r"((uint32_t)kTcRows)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void tc_group_sync(uint32_t g) {
    asm volatile("bar.sync %0, %1;" ::"r"(1u + g), "r"((uint32_t)kTcRows) : "memory");
}

// 16 f32 accumulator columns of this thread's row (lane = row within the warp's 32).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// The 64 bias values of a layer into this thread's row of the accumulators.
__device__ __forceinline__ void tc_st_bias(uint32_t taddr, const float* bias) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float4* b = reinterpret_cast<const float4*>(bias + 16 * c);
        const float4 q0 = b[0], q1 = b[1], q2 = b[2], q3 = b[3];
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16};" ::"r"(taddr + 16u * c),
            "f"(q0.x), "f"(q0.y), "f"(q0.z), "f"(q0.w), "f"(q1.x), "f"(q1.y), "f"(q1.z), "f"(q1.w), "f"(q2.x),
            "f"(q2.y), "f"(q2.z), "f"(q2.w), "f"(q3.x), "f"(q3.y), "f"(q3.z), "f"(q3.w)
            : "memory");
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(kTcThreads, kTcBlocksPerSM)
    k_fsai_infer_tc(FeatCtx fc, const float* __restrict__ P, float* __restrict__ g, uint32_t* __restrict__ words) {
    extern __shared__ __align__(128) unsigned char tc_raw[];
    TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_raw);
    const uint32_t tid = threadIdx.x, gi = tid / kTcRows, r = tid % kTcRows, w = tid >> 5;
    TcGroupSmem& gs = sm.grp[gi];
    // weights as W^T (N x K, K-major), bf16 rounded like the mma.sync fragments
    for (uint32_t t = tid; t < (uint32_t)(kFsaiHid * kFsaiNF); t += kTcThreads) {
        const uint32_t n = t % kFsaiHid, k = t / kFsaiHid;
        sm.B1[tc_idx(n, k, 2)] = __float2bfloat16_rn(P[kOffW1 + k * kFsaiHid + n]);
    }
    for (uint32_t t = tid; t < (uint32_t)(kFsaiHid * kFsaiHid); t += kTcThreads) {
        const uint32_t n = t % kFsaiHid, k = t / kFsaiHid;
        sm.B2[tc_idx(n, k, 8)] = __float2bfloat16_rn(P[kOffW2 + k * kFsaiHid + n]);
        sm.B3[tc_idx(n, k, 8)] = __float2bfloat16_rn(P[kOffW3 + k * kFsaiHid + n]);
    }
    for (uint32_t t = tid; t < (uint32_t)kFsaiHid; t += kTcThreads) {
        sm.bias[0][t] = P[kOffB1 + t];
        sm.bias[1][t] = P[kOffB2 + t];
        sm.bias[2][t] = P[kOffB3 + t];
        sm.w4[t] = round_bf16(P[kOffW4 + t]);
    }
    if (tid == 0) {
        sm.b4 = P[kOffB4];
        for (int q = 0; q < kTcGroups; ++q)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(&sm.mbar[q]))
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (w == 0) {  // tensor memory for every group's 128 x 64 accumulators (warp 0 allocates and frees)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(&sm.tmem)),
                     "r"(kTcAlloc)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = sm.tmem + kTcCols * gi;             // the group's columns
    const uint32_t trow = tbase + ((32u * (w & 3u)) << 16);    // this warp's 32 lanes
    uint64_t* bar = &sm.mbar[gi];
    const uint64_t dB1 = tc_desc(sm.B1, 128, 256), dA1 = tc_desc(gs.A1, 128, 256);
    uint32_t phase = 0;
    bool issued = false, failed = false;
    tc_st_bias(trow, sm.bias[0]);
    const uint32_t n_tiles = (fc.n_edges + kTcRows - 1) / kTcRows;
    for (uint32_t tile = blockIdx.x * kTcGroups + gi; tile < n_tiles && !failed; tile += gridDim.x * kTcGroups) {
        const uint32_t e = tile * kTcRows + r;
        EdgeInfo info;
        float f[kFsaiNF];
        if (e < fc.n_edges) {
            edge_features(fc, e, f, info);
        } else {
#pragma unroll
            for (int t = 0; t < kFsaiNF; ++t) f[t] = 0.f;
            info = EdgeInfo{0u, 0.f, 3u, 0.f};
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            uint32_t wv[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) wv[q] = pack_bf16(f[8 * c + 2 * q], f[8 * c + 2 * q + 1]);
            *reinterpret_cast<uint4*>(&gs.A1[tc_idx(r, 8 * c, 2)]) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
        }
        float out = 0.f;
        for (int layer = 0; layer < 3; ++layer) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic smem writes -> tensor core
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            tc_group_sync(gi);
            if (r == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (layer == 0) {
                    tc_mma(tbase, dA1, dB1, 1u);
                } else {
                    const __nv_bfloat16* B = layer == 1 ? sm.B2 : sm.B3;
#pragma unroll
                    for (uint32_t j = 0; j < 4; ++j)  // K = 64 as four K = 16 steps: core-matrix columns 2j, 2j + 1
                        tc_mma(tbase, tc_desc(gs.A2 + j * 128, 128, 1024), tc_desc(B + j * 128, 128, 1024), 1u);
                }
                tc_commit(bar);
            }
            issued = true;
            const bool ok = tc_wait(bar, phase);
            if (tc_group_sync_or(gi, !ok)) {  // uniform over the group
                failed = true;
                break;
            }
            issued = false;
            phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int h = 0; h < 4; ++h) {  // 16 columns at a time
                float z[16];
                tc_ld16(trow + 16u * h, z);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (layer < 2) {
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        uint32_t wv[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) wv[q] = pack_bf16(gelu(z[8 * c + 2 * q]), gelu(z[8 * c + 2 * q + 1]));
                        *reinterpret_cast<uint4*>(&gs.A2[tc_idx(r, 16 * h + 8 * c, 8)]) =
                            make_uint4(wv[0], wv[1], wv[2], wv[3]);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) out += gelu(z[i]) * sm.w4[16 * h + i];
                }
            }
            tc_st_bias(trow, sm.bias[layer < 2 ? layer + 1 : 0]);  // the next layer's (or tile's) start
        }
        if (failed) break;
        if (info.kind != 3) g[info.pos] = g_value(info, sm.b4 + out);
    }
    if (failed) {
        if (r == 0) atomicOr(words, kErrTensorWait);
        if (issued) tc_wait(bar, phase);  // the last commit before freeing its accumulators (bounded)
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem), "r"(kTcAlloc)
                     : "memory");
    }
}

}  // namespace

FsaiModel::FsaiModel() {
    params.ensure(kFsaiParamCount);
    grad.ensure(kFsaiParamCount);
    gsum.ensure(kFsaiParamCount);
    m.ensure(kFsaiParamCount);
    v.ensure(kFsaiParamCount);
    frags.ensure(kFragCount);
    acc.ensure(2);
    SB_CUDA(cudaMemset(params.ptr, 0, sizeof(float) * kFsaiParamCount));
    SB_CUDA(cudaMemset(grad.ptr, 0, sizeof(float) * kFsaiParamCount));
    SB_CUDA(cudaMemset(m.ptr, 0, sizeof(float) * kFsaiParamCount));
    SB_CUDA(cudaMemset(v.ptr, 0, sizeof(float) * kFsaiParamCount));
}

void FsaiModel::pack(cudaStream_t s) {
    k_fsai_pack<<<grid_for(kFragCount, 256), 256, 0, s>>>(params.ptr, frags.ptr);
    SB_LAUNCH_CHECK();
    packed = true;
}

void fsai_prepare(const CsrF64& A, const float4* xyz, FsaiSystem& S, cudaStream_t s) {
    const uint32_t n = A.n;
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, s));
    S.n = n;
    S.nnz = A.nnz;
    S.dpos.ensure(n);
    S.lcnt.ensure(n);
    S.loff.ensure((size_t)n + 1);
    S.node.ensure(n);
    S.red.ensure(4);
    S.words.ensure(4);
    SB_CUDA(cudaMemsetAsync(S.red.ptr, 0, 4 * sizeof(double), s));
    SB_CUDA(cudaMemsetAsync(S.words.ptr, 0, 4 * sizeof(uint32_t), s));
    k_fsai_rows<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, A.row.ptr, A.col.ptr, A.val.ptr, xyz, S.dpos.ptr,
                                                           S.lcnt.ptr, S.node.ptr, S.red.ptr, S.words.ptr);
    SB_LAUNCH_CHECK();
    exclusive_scan_u32(S.scan, S.lcnt.ptr, S.loff.ptr, n, s);
    double red[4];
    uint32_t ne = 0, err = 0;
    SB_CUDA(cudaMemcpyAsync(red, S.red.ptr, sizeof red, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaMemcpyAsync(&ne, S.loff.ptr + n, sizeof ne, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaMemcpyAsync(&err, S.words.ptr, sizeof err, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    S.n_edges = ne;
    S.error = err;
    const double lmean = red[1] > 0 ? red[0] / red[1] : 0.0;
    S.inv_h = (xyz && red[3] > 0 && red[2] > 0) ? (float)(red[3] / red[2]) : 1.f;
    k_fsai_nodes<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, S.dpos.ptr, A.val.ptr, lmean, S.node.ptr);
    SB_LAUNCH_CHECK();
    S.e_row.ensure(ne);
    S.e_pos.ensure(ne);
    k_fsai_edges<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, A.row.ptr, S.loff.ptr, S.e_row.ptr, S.e_pos.ptr);
    SB_LAUNCH_CHECK();
    S.g.ensure(A.nnz);
    if (!S.error) {  // compact patterns of the two halves
        S.lcol.ensure(ne);
        if (ne) {
            k_fsai_lower_cols<<<grid_for(ne, kThreads), kThreads, 0, s>>>(ne, S.e_pos.ptr, A.col.ptr, S.lcol.ptr);
            SB_LAUNCH_CHECK();
        }
        S.ucnt.ensure(n);
        S.uoff.ensure((size_t)n + 1);
        k_fsai_upper_cnt<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, A.row.ptr, S.dpos.ptr, S.ucnt.ptr);
        SB_LAUNCH_CHECK();
        exclusive_scan_u32(S.scan, S.ucnt.ptr, S.uoff.ptr, n, s);
        SB_CUDA(cudaMemcpyAsync(&S.n_upper, S.uoff.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SB_CUDA(cudaStreamSynchronize(s));
        S.ucol.ensure(S.n_upper);
        k_fsai_upper_fill<<<grid_for(n, kThreads), kThreads, 0, s>>>(n, S.dpos.ptr, S.uoff.ptr, A.col.ptr, nullptr,
                                                                     S.ucol.ptr, nullptr, nullptr);
        SB_LAUNCH_CHECK();
    }
    SB_CUDA(cudaEventRecord(e1, s));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    S.setup_ms = ms;
    S.prepared = true;
    S.g_model = nullptr;
    S.g_version = 0;
}

namespace {
// The upper half of g mirrored from the lower one, and the solver's FP16
// copies of both halves.
void build_operator(const CsrF64& A, FsaiSystem& S, cudaStream_t s) {
    k_fsai_mirror<<<grid_for(S.n, kThreads), kThreads, 0, s>>>(S.n, A.row.ptr, A.col.ptr, S.dpos.ptr, S.g.ptr,
                                                               S.words.ptr);
    SB_LAUNCH_CHECK();
    S.gmax.ensure(1);
    absmax_f32(S.g.ptr, S.nnz, S.gmax.ptr, s);
    S.lval.ensure(S.n_edges);
    S.uval.ensure(S.n_upper);
    if (S.n_edges) {
        k_fsai_lower_vals<<<grid_for(S.n_edges, kThreads), kThreads, 0, s>>>(S.n_edges, S.e_pos.ptr, S.g.ptr,
                                                                              S.gmax.ptr, S.lval.ptr);
        SB_LAUNCH_CHECK();
    }
    k_fsai_upper_fill<<<grid_for(S.n, kThreads), kThreads, 0, s>>>(S.n, S.dpos.ptr, S.uoff.ptr, nullptr, S.g.ptr,
                                                                   nullptr, S.gmax.ptr, S.uval.ptr);
    SB_LAUNCH_CHECK();
}
}  // namespace

namespace {
// The Kolotilina-Yeremin G into dst (aligned with A's entries, lower halves
// written); the status words are cleared first and words[1] counts the rows
// left diagonal.
void launch_ky(const CsrF64& A, FsaiSystem& S, float* dst, cudaStream_t s) {
    SB_CUDA(cudaMemsetAsync(S.words.ptr, 0, 4 * sizeof(uint32_t), s));
    k_fsai_ky<<<grid_for(S.n, 128), 128, 0, s>>>(S.n, A.row.ptr, A.col.ptr, A.val.ptr, S.dpos.ptr, dst,
                                                 S.words.ptr);
    SB_LAUNCH_CHECK();
}
// The base G of a KY-based model on this system (once per matrix).
void ensure_ky_base(const CsrF64& A, FsaiSystem& S, cudaStream_t s) {
    if (S.ky_ready) return;
    S.ky.ensure(S.nnz);
    launch_ky(A, S, S.ky.ptr, s);
    uint32_t rows = 0;
    SB_CUDA(cudaMemcpyAsync(&rows, S.words.ptr + 1, sizeof rows, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    S.ky_diag_rows = rows;
    S.ky_ready = true;
}
}  // namespace

void fsai_ky(const CsrF64& A, const float4* xyz, FsaiSystem& S, cudaStream_t s) {
    if (!S.prepared) fsai_prepare(A, xyz, S, s);
    if (S.error) throw std::runtime_error("fsai: the matrix needs a positive diagonal and sorted columns");
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, s));
    launch_ky(A, S, S.g.ptr, s);
    build_operator(A, S, s);
    SB_CUDA(cudaEventRecord(e1, s));
    uint32_t w2[2] = {0, 0};
    SB_CUDA(cudaMemcpyAsync(w2, S.words.ptr, sizeof w2, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaEventSynchronize(e1));
    SB_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    S.infer_ms = ms;
    S.error = w2[0];
    S.ky_diag_rows = w2[1];
    if (w2[0]) throw std::runtime_error("fsai: the matrix pattern is not symmetric");
    S.g_model = nullptr;
    S.g_version = 0;
    S.g_ky = true;
}

void fsai_infer(FsaiModel& M, const CsrF64& A, const float4* xyz, FsaiSystem& S, cudaStream_t s) {
    if (!S.prepared) fsai_prepare(A, xyz, S, s);
    if (S.error) throw std::runtime_error("fsai: the matrix needs a positive diagonal and sorted columns");
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    SB_CUDA(cudaEventRecord(e0, s));
    const bool ky = M.base == kFsaiBaseKy;
    if (ky) ensure_ky_base(A, S, s);
    if (S.n_edges) {
        static_assert(kTcBlocksPerSM * (sizeof(TcSmem) + 1024) <= 228 * 1024, "resident blocks fit shared memory");
        static std::atomic<uint64_t> attr{0};  // one bit per device
        if (once_per_device(attr))
            SB_CUDA(cudaFuncSetAttribute(k_fsai_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(TcSmem)));
        const uint32_t tiles = (S.n_edges + kTcRows - 1) / kTcRows;
        k_fsai_infer_tc<<<mlp_grid(tiles, kTcGroups, kNumSMs * kTcBlocksPerSM), kTcThreads, sizeof(TcSmem), s>>>(
            feat_ctx(A, xyz, S, ky), M.params.ptr, S.g.ptr, S.words.ptr);
        SB_LAUNCH_CHECK();
    }
    build_operator(A, S, s);
    SB_CUDA(cudaEventRecord(e1, s));
    uint32_t err = 0;
    SB_CUDA(cudaMemcpyAsync(&err, S.words.ptr, sizeof err, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaEventSynchronize(e1));
    SB_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    S.infer_ms = ms;
    S.error = err;
    if (err & kErrTensorWait) throw std::runtime_error("fsai: a tensor-core completion wait timed out");
    if (err) throw std::runtime_error("fsai: the matrix pattern is not symmetric");
    S.g_model = &M;
    S.g_version = M.version;
    S.g_ky = false;
}

void fsai_features(const CsrF64& A, const float4* xyz, FsaiSystem& S, float* out, cudaStream_t s, bool ky) {
    if (!S.prepared) fsai_prepare(A, xyz, S, s);
    if (ky) ensure_ky_base(A, S, s);
    if (S.n_edges) {
        k_fsai_features<<<grid_for(S.n_edges, kThreads), kThreads, 0, s>>>(feat_ctx(A, xyz, S, ky), out);
        SB_LAUNCH_CHECK();
    }
}

double fsai_loss_grad(FsaiModel& M, const CsrF64& A, const float4* xyz, FsaiSystem& S, uint64_t seed,
                      const float* z_host, cudaStream_t s) {
    M.pack(s);
    fsai_infer(M, A, xyz, S, s);
    const uint32_t n = S.n;
    const size_t nb = (size_t)n * kFsaiProbes;
    S.Z.ensure(nb); S.Y.ensure(nb); S.W.ensure(nb); S.E.ensure(nb); S.T.ensure(nb);
    S.dG.ensure(S.n_edges);
    if (z_host) SB_CUDA(cudaMemcpyAsync(S.Z.ptr, z_host, sizeof(float) * nb, cudaMemcpyHostToDevice, s));
    else {
        k_fsai_probes<<<grid_for(nb, kThreads), kThreads, 0, s>>>(n, seed, S.Z.ptr);
        SB_LAUNCH_CHECK();
    }
    SB_CUDA(cudaMemsetAsync(M.acc.ptr, 0, 2 * sizeof(double), s));
    const int gs = grid_for(nb, kThreads);
    const uint32_t *row = A.row.ptr, *col = A.col.ptr, *dp = S.dpos.ptr;
    if (M.loss_kind == kFsaiLossKaporin) {
        // Y = G^T Z ; W = A Y with acc[0] = sum Y.W ; acc[1] = sum log G_ii
        k_fsai_spmm<2><<<gs, kThreads, 0, s>>>(n, row, col, dp, A.val.ptr, S.g.ptr, S.Z.ptr, S.Y.ptr, nullptr,
                                               nullptr);
        SB_LAUNCH_CHECK();
        k_fsai_spmm<3><<<gs, kThreads, 0, s>>>(n, row, col, dp, A.val.ptr, S.g.ptr, S.Y.ptr, S.W.ptr, nullptr,
                                               M.acc.ptr);
        SB_LAUNCH_CHECK();
        k_fsai_logdiag<<<std::min(grid_for(n, kThreads), kNumSMs * 4), kThreads, 0, s>>>(n, dp, S.g.ptr, M.acc.ptr);
        SB_LAUNCH_CHECK();
        if (S.n_edges) {
            k_fsai_dG_kaporin<<<grid_for((size_t)S.n_edges * kFsaiProbes, kThreads), kThreads, 0, s>>>(
                n, S.n_edges, S.e_row.ptr, S.e_pos.ptr, col, S.Z.ptr, S.W.ptr, S.g.ptr, M.acc.ptr, S.dG.ptr);
            SB_LAUNCH_CHECK();
        }
    } else {  // residual
        // Y = G^T Z ; W = A Y ; E = G W - Z ; U = G^T E (into Y) ; T = A U
        const double* av = A.val.ptr;
        const float* g = S.g.ptr;
        k_fsai_spmm<2><<<gs, kThreads, 0, s>>>(n, row, col, dp, av, g, S.Z.ptr, S.Y.ptr, nullptr, nullptr);
        SB_LAUNCH_CHECK();
        k_fsai_spmm<0><<<gs, kThreads, 0, s>>>(n, row, col, dp, av, g, S.Y.ptr, S.W.ptr, nullptr, nullptr);
        SB_LAUNCH_CHECK();
        k_fsai_spmm<1><<<gs, kThreads, 0, s>>>(n, row, col, dp, av, g, S.W.ptr, S.E.ptr, S.Z.ptr, M.acc.ptr);
        SB_LAUNCH_CHECK();
        k_fsai_spmm<2><<<gs, kThreads, 0, s>>>(n, row, col, dp, av, g, S.E.ptr, S.Y.ptr, nullptr, nullptr);
        SB_LAUNCH_CHECK();
        k_fsai_spmm<0><<<gs, kThreads, 0, s>>>(n, row, col, dp, av, g, S.Y.ptr, S.T.ptr, nullptr, nullptr);
        SB_LAUNCH_CHECK();
        const float scale = (float)(2.0 / ((double)kFsaiProbes * n));
        if (S.n_edges) {
            k_fsai_dG<<<grid_for((size_t)S.n_edges * kFsaiProbes, kThreads), kThreads, 0, s>>>(
                S.n_edges, S.e_row.ptr, S.e_pos.ptr, col, S.E.ptr, S.W.ptr, S.Z.ptr, S.T.ptr, scale, S.dG.ptr);
            SB_LAUNCH_CHECK();
        }
    }
    const int nblk = mlp_grid(S.n_edges, kTrainEdges, kNumSMs * 2);
    M.partials.ensure((size_t)nblk * kFsaiParamCount);
    SB_CUDA(cudaFuncSetAttribute(k_fsai_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem)));
    k_fsai_train<<<nblk, kMlpThreads, sizeof(TrainSmem), s>>>(feat_ctx(A, xyz, S, M.base == kFsaiBaseKy),
                                                              M.params.ptr, M.frags.ptr, S.dG.ptr,
                                                               M.partials.ptr);
    SB_LAUNCH_CHECK();
    k_fsai_reduce<<<grid_for(kFsaiParamCount, 256), 256, 0, s>>>(M.partials.ptr, (uint32_t)nblk, M.grad.ptr);
    SB_LAUNCH_CHECK();
    double acc[2] = {0.0, 0.0};
    SB_CUDA(cudaMemcpyAsync(acc, M.acc.ptr, sizeof acc, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (M.loss_kind == kFsaiLossKaporin) return std::log(acc[0] / ((double)kFsaiProbes * n)) - 2.0 / n * acc[1];
    return acc[0] / ((double)kFsaiProbes * n);
}

void fsai_accumulate(FsaiModel& M, float w, bool first, bool last, cudaStream_t s) {
    k_fsai_accumulate<<<grid_for(kFsaiParamCount, 256), 256, 0, s>>>(M.gsum.ptr, M.grad.ptr, w, first ? 1 : 0,
                                                                     last ? 1 : 0);
    SB_LAUNCH_CHECK();
}

void fsai_adam(FsaiModel& M, float lr, float clip, cudaStream_t s) {
    ++M.adam_t;
    const float bc1 = 1.f - std::pow(0.9f, (float)M.adam_t), bc2 = 1.f - std::pow(0.999f, (float)M.adam_t);
    k_fsai_adam<<<1, 1024, 0, s>>>(M.params.ptr, M.grad.ptr, M.m.ptr, M.v.ptr, lr, bc1, bc2, clip);
    SB_LAUNCH_CHECK();
    ++M.version;
    M.packed = false;
}

}  // namespace sb
