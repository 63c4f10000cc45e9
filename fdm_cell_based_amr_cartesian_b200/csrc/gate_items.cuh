// gate_items.cuh — inference side of the learned face gate, shared by the
// single-mesh kernels (gate.cu) and the batched persistent kernel
// (batch.cu): the features of a face stencil, the linear-weight flux, the
// BF16 MLP on the tensor cores (mma.sync.m16n8k16, FP32 accumulation), and
// the per-warp work of the stage-1 gate and the stage-2/3 guard.  No
// reference counterpart: the reference always evaluates the nonlinear
// weights (src/nnd_center_RK.F90:310-353).
#pragma once

#include <cuda_bf16.h>

#include "items.cuh"

namespace fdm {

constexpr int GF = 8;    // features
constexpr int GH = 32;   // hidden width
// parameter block (FP32): W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3
constexpr int P_W1 = 0, P_B1 = P_W1 + GH * GF, P_W2 = P_B1 + GH, P_B2 = P_W2 + GH * GH, P_W3 = P_B2 + GH,
              P_B3 = P_W3 + GH, P_N = P_B3 + 1;   // 1377

// ----------------------------------------------------------- features
__device__ __forceinline__ float squash(float x) {
    // sign(x) * log10(1 + 1e4 |x|) / 4: 1e-4 -> 0.08, 1e-2 -> 0.5, 1 -> 1
    // (hardware log2; log10(2)/4 = 0.0752574989)
    const float v = __log2f(1.0f + 1.0e4f * fabsf(x)) * 0.0752574989f;
    return x < 0.f ? -v : v;
}
// 8 features of a face stencil s0..s3 (FP32; the network reads BF16):
// jumps of rho and p normalised by the face means, largest normal and
// tangential velocity jump over the face sound speed
// (jump) receives the largest of the unsquashed feature magnitudes.
template <int DIR>
__device__ __forceinline__ void face_features(const Prim &s0, const Prim &s1, const Prim &s2, const Prim &s3,
                                              double g, float f[GF], float *jump = nullptr) {
    const float rs = (float)(s1.r + s2.r), ps = (float)(s1.p + s2.p);
    const float irb = __fdividef(2.0f, rs), ipb = __fdividef(2.0f, ps);
    const float ic = rsqrtf(fabsf((float)g * ps / rs) + 1e-30f);
    const Prim P[4] = {s0, s1, s2, s3};
    float dun = 0.f, dut = 0.f, jm = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float jr = (float)(P[k + 1].r - P[k].r) * irb, jp = (float)(P[k + 1].p - P[k].p) * ipb;
        jm = fmaxf(jm, fmaxf(fabsf(jr), fabsf(jp)));
        f[k] = squash(jr);
        f[3 + k] = squash(jp);
        const double un0 = DIR == 0 ? P[k].u : P[k].v, un1 = DIR == 0 ? P[k + 1].u : P[k + 1].v;
        const double ut0 = DIR == 0 ? P[k].v : P[k].u, ut1 = DIR == 0 ? P[k + 1].v : P[k + 1].u;
        dun = fmaxf(dun, fabsf((float)(un1 - un0)));
        dut = fmaxf(dut, fabsf((float)(ut1 - ut0)));
    }
    f[6] = squash(dun * ic);
    f[7] = squash(dut * ic);
    if (jump) *jump = fmaxf(jm, fmaxf(dun, dut) * ic);
}

// The same largest jump without the features (stages 2 and 3).
template <int DIR>
__device__ __forceinline__ float face_jump(const Prim &s0, const Prim &s1, const Prim &s2, const Prim &s3, double g) {
    const float rs = (float)(s1.r + s2.r), ps = (float)(s1.p + s2.p);
    const float irb = __fdividef(2.0f, rs), ipb = __fdividef(2.0f, ps);
    const float ic = rsqrtf(fabsf((float)g * ps / rs) + 1e-30f);
    const Prim P[4] = {s0, s1, s2, s3};
    float jm = 0.f, dv = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        jm = fmaxf(jm, fabsf((float)(P[k + 1].r - P[k].r) * irb));
        jm = fmaxf(jm, fabsf((float)(P[k + 1].p - P[k].p) * ipb));
        dv = fmaxf(dv, fabsf((float)(P[k + 1].u - P[k].u)));
        dv = fmaxf(dv, fabsf((float)(P[k + 1].v - P[k].v)));
    }
    return fmaxf(jm, dv * ic);
}

// Effect of the nonlinear weight of one WCNS_Z3 reconstruction: with
// w2 = 1 - w1 the nonlinear value differs from the linear-weight value by
// exactly (w1 - l1) (p1 - p2), l1 = d1/(d1+d2) the normalised linear weight.
__device__ __forceinline__ double wcns_effect(double u1, double u2, double u3) {
    const double d1 = FDM_D1_WCNS, d2 = FDM_D2_WCNS;
    double t = -u1 + u2;
    double IS1 = t * t;
    t = -u2 + u3;
    const double IS2a = t * t;
    t = u1 - 2. * u2 + u3;
    const double IS3 = t * t;
    const double p1 = u2;
    const double p2 = ((-u1 + 6.0 * u2 + 3.0 * u3) / 8.0 - d1 * p1) / d2;
    IS1 = fmin(IS1, IS2a);
    const double IS2 = IS3 + u1 * u1 + u2 * u2 + u3 * u3 - u1 * u2 - u2 * u3 - u1 * u3;
    t = 10. * fabs(IS2 - 3. * IS1);
    const double tau3 = t * t;
    const double a1 = d1 * (1.0 + tau3 / (FDM_EPS_WCNS + IS1));
    const double a2 = d2 * (1.0 + tau3 / (FDM_EPS_WCNS + IS2));
    const double w1 = a1 / (a1 + a2), l1 = d1 / (d1 + d2);
    return fabs(w1 - l1) * fabs(p1 - p2);
}
// Largest relative effect over the 16 WCNS_Z3 reconstructions of a face:
// per characteristic component, the effect over the component's largest
// magnitude on the 4-point stencil.
template <int DIR>
__device__ double face_weight_deviation(const Prim &s0, const Prim &s1, const Prim &s2, const Prim &s3, double g) {
    double U[4][4], F[4][4];
    cons_flux<DIR>(s0, g, U[0], F[0]);
    cons_flux<DIR>(s1, g, U[1], F[1]);
    cons_flux<DIR>(s2, g, U[2], F[2]);
    cons_flux<DIR>(s3, g, U[3], F[3]);
    double Um[4];
    for (int r = 0; r < 4; ++r) Um[r] = (U[1][r] + U[2][r]) / 2.0;
    Eig E;
    eigen<DIR>(Um, g, E);
    double w[4][4], q[4][4];
    for (int k = 0; k < 4; ++k) { project<DIR>(E, U[k], w[k]); project<DIR>(E, F[k], q[k]); }
    double dev = 0.0;
    for (int r = 0; r < 4; ++r) {
        const double sw = fmax(fmax(fabs(w[0][r]), fabs(w[1][r])), fmax(fabs(w[2][r]), fabs(w[3][r]))) + 1e-300;
        const double sq = fmax(fmax(fabs(q[0][r]), fabs(q[1][r])), fmax(fabs(q[2][r]), fabs(q[3][r]))) + 1e-300;
        dev = fmax(dev, wcns_effect(w[0][r], w[1][r], w[2][r]) / sw);
        dev = fmax(dev, wcns_effect(w[3][r], w[2][r], w[1][r]) / sw);
        dev = fmax(dev, wcns_effect(q[0][r], q[1][r], q[2][r]) / sq);
        dev = fmax(dev, wcns_effect(q[3][r], q[2][r], q[1][r]) / sq);
    }
    return dev;
}

// Linear-weight flux: with linear weights the characteristic projection
// cancels (R Ri = I), so the reconstruction is component-wise on the
// conserved variables and fluxes: ((-u0 + 6 u1 + 3 u2)/8) / (d1 + d2), the
// REAL(4) pair d1, d2 kept.  ig1 = 1/(gamma-1), c8 = 1/(8 (d1+d2)).
template <int DIR>
__device__ __forceinline__ void cons_flux_lin(const Prim &q, double ig1, double U[4], double F[4]) {
    const double ke = q.u * q.u + q.v * q.v;
    const double E = q.p * ig1 + 0.5 * q.r * ke;
    const double un = DIR == 0 ? q.u : q.v;
    U[0] = q.r;
    U[1] = q.r * q.u;
    U[2] = q.r * q.v;
    U[3] = E;
    F[0] = q.r * un;
    F[1] = U[1] * un + (DIR == 0 ? q.p : 0.0);
    F[2] = U[2] * un + (DIR == 0 ? 0.0 : q.p);
    F[3] = un * (E + q.p);
}
template <int DIR>
__device__ __forceinline__ void face_flux_linear(const Prim &s0, const Prim &s1, const Prim &s2, const Prim &s3,
                                                 double ig1, double lam, double out[4]) {
    double U[4][4], F[4][4];
    cons_flux_lin<DIR>(s0, ig1, U[0], F[0]);
    cons_flux_lin<DIR>(s1, ig1, U[1], F[1]);
    cons_flux_lin<DIR>(s2, ig1, U[2], F[2]);
    cons_flux_lin<DIR>(s3, ig1, U[3], F[3]);
    const double c8 = 1.0 / (8.0 * (FDM_D1_WCNS + FDM_D2_WCNS));
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const double wL = (-U[0][r] + 6.0 * U[1][r] + 3.0 * U[2][r]) * c8;
        const double wR = (-U[3][r] + 6.0 * U[2][r] + 3.0 * U[1][r]) * c8;
        const double gL = (-F[0][r] + 6.0 * F[1][r] + 3.0 * F[2][r]) * c8;
        const double gR = (-F[3][r] + 6.0 * F[2][r] + 3.0 * F[1][r]) * c8;
        out[r] = 0.5 * (gL + gR - lam * (wR - wL));
    }
}

// ------------------------------------------------------- tensor-core MLP
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat16 a = __float2bfloat16_rn(lo), b = __float2bfloat16_rn(hi);
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// D = A(16x16 bf16, row) * B(16x8 bf16, col) + C (f32)
__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], const uint32_t b[2], const float c[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%10,%11,%12,%13};\n"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "f"(c[0]), "f"(c[1]), "f"(c[2]),
          "f"(c[3]));
}

// hardware tanh (MUFU, relative error ~2^-11, below the BF16 rounding of
// the activations it feeds)
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu(float x) {
    const float k = 0.7978845608028654f;
    const float t = tanh_fast(k * (x + 0.044715f * x * x * x));
    return 0.5f * x * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float k = 0.7978845608028654f;
    const float t = tanh_fast(k * (x + 0.044715f * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k * (1.0f + 3.0f * 0.044715f * x * x);
}

// Shared-memory row pitches (bf16 elements), padded so that the fragment
// reads of a warp (rows g = lane/4, word t = lane%4) hit distinct banks.
constexpr int XLD = 24, HLD = 40;

// BF16 weights in the layout the fragments read
struct __align__(16) GateWeights {
    __nv_bfloat16 W1[GH][XLD];   // [out][in], inputs 8.. zero
    __nv_bfloat16 W2[GH][HLD];   // [out][in]
    __nv_bfloat16 w3[GH];
    float b1[GH], b2[GH], b3;
};

// Per-warp staging of the 32 feature rows for inference
struct __align__(16) XTile {
    __nv_bfloat16 X[32][XLD];   // columns GF.. stay zero
};

// Per-warp staging of 32 samples (rows) in shared memory; rows of X are
// written as one 16-byte vector per lane (row pitch 48 bytes)
struct __align__(16) WarpTile {
    __nv_bfloat16 X[32][XLD];   // columns GF.. stay zero
    __nv_bfloat16 H1[32][HLD];
    __nv_bfloat16 H2[32][HLD];
};

// A fragment (rows m0..m0+15, cols k0..k0+15) of a row-major bf16 tile
template <int LD>
__device__ __forceinline__ void load_a(const __nv_bfloat16 (*M)[LD], int m0, int k0, uint32_t a[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int r0 = m0 + g, r1 = m0 + g + 8, c0 = k0 + 2 * t, c1 = k0 + 2 * t + 8;
    a[0] = (uint32_t)__bfloat16_as_ushort(M[r0][c0]) | ((uint32_t)__bfloat16_as_ushort(M[r0][c0 + 1]) << 16);
    a[1] = (uint32_t)__bfloat16_as_ushort(M[r1][c0]) | ((uint32_t)__bfloat16_as_ushort(M[r1][c0 + 1]) << 16);
    a[2] = (uint32_t)__bfloat16_as_ushort(M[r0][c1]) | ((uint32_t)__bfloat16_as_ushort(M[r0][c1 + 1]) << 16);
    a[3] = (uint32_t)__bfloat16_as_ushort(M[r1][c1]) | ((uint32_t)__bfloat16_as_ushort(M[r1][c1 + 1]) << 16);
}
// B fragment for D = A * W^T with W [out][in] row-major: B[k][n] = W[n0+n][k0+k]
template <int LD>
__device__ __forceinline__ void load_b_wt(const __nv_bfloat16 (*W)[LD], int n0, int k0, uint32_t b[2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int n = n0 + g, k = k0 + 2 * t;
    b[0] = (uint32_t)__bfloat16_as_ushort(W[n][k]) | ((uint32_t)__bfloat16_as_ushort(W[n][k + 1]) << 16);
    b[1] = (uint32_t)__bfloat16_as_ushort(W[n][k + 8]) | ((uint32_t)__bfloat16_as_ushort(W[n][k + 9]) << 16);
}

// Forward pass of 32 samples staged in T.X; pre-activations a1, a2 and the
// logits z (per row) are returned, h1 / h2 are left in T.H1 / T.H2.
// Layouts: acc[mt][nt][i] is row mt*16 + g + 8*(i>>1), col nt*8 + 2t + (i&1).
__device__ __forceinline__ void mlp_forward(const GateWeights &W, WarpTile &T, float a1[2][4][4], float a2[2][4][4],
                                            float z[2][2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int mt = 0; mt < 2; ++mt) {
        uint32_t a[4];
        load_a<XLD>(T.X, mt * 16, 0, a);
        for (int nt = 0; nt < 4; ++nt) {
            uint32_t b[2];
            load_b_wt<XLD>(W.W1, nt * 8, 0, b);
            const float c[4] = {W.b1[nt * 8 + 2 * t], W.b1[nt * 8 + 2 * t + 1], W.b1[nt * 8 + 2 * t],
                                W.b1[nt * 8 + 2 * t + 1]};
            mma16816(a1[mt][nt], a, b, c);
        }
        for (int nt = 0; nt < 4; ++nt)
            for (int i = 0; i < 4; ++i)
                T.H1[mt * 16 + g + 8 * (i >> 1)][nt * 8 + 2 * t + (i & 1)] = __float2bfloat16_rn(gelu(a1[mt][nt][i]));
    }
    __syncwarp();
    for (int mt = 0; mt < 2; ++mt) {
        for (int nt = 0; nt < 4; ++nt) {
            float c[4] = {W.b2[nt * 8 + 2 * t], W.b2[nt * 8 + 2 * t + 1], W.b2[nt * 8 + 2 * t],
                          W.b2[nt * 8 + 2 * t + 1]};
            for (int kc = 0; kc < 2; ++kc) {
                uint32_t a[4], b[2];
                load_a<HLD>(T.H1, mt * 16, kc * 16, a);
                load_b_wt<HLD>(W.W2, nt * 8, kc * 16, b);
                float d[4];
                mma16816(d, a, b, c);
                c[0] = d[0]; c[1] = d[1]; c[2] = d[2]; c[3] = d[3];
            }
            for (int i = 0; i < 4; ++i) a2[mt][nt][i] = c[i];
        }
        for (int nt = 0; nt < 4; ++nt)
            for (int i = 0; i < 4; ++i)
                T.H2[mt * 16 + g + 8 * (i >> 1)][nt * 8 + 2 * t + (i & 1)] = __float2bfloat16_rn(gelu(a2[mt][nt][i]));
    }
    __syncwarp();
    // layer 3: N padded to 8, only column 0 is w3
    for (int mt = 0; mt < 2; ++mt) {
        float c[4] = {W.b3, 0.f, W.b3, 0.f};
        for (int kc = 0; kc < 2; ++kc) {
            uint32_t a[4], b[2];
            load_a<HLD>(T.H2, mt * 16, kc * 16, a);
            const int k = kc * 16 + 2 * t;
            const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
            const __nv_bfloat16 w0 = g == 0 ? W.w3[k] : zero, w1 = g == 0 ? W.w3[k + 1] : zero;
            const __nv_bfloat16 w8 = g == 0 ? W.w3[k + 8] : zero, w9 = g == 0 ? W.w3[k + 9] : zero;
            b[0] = (uint32_t)__bfloat16_as_ushort(w0) | ((uint32_t)__bfloat16_as_ushort(w1) << 16);
            b[1] = (uint32_t)__bfloat16_as_ushort(w8) | ((uint32_t)__bfloat16_as_ushort(w9) << 16);
            float d[4];
            mma16816(d, a, b, c);
            c[0] = d[0]; c[1] = d[1]; c[2] = d[2]; c[3] = d[3];
        }
        z[mt][0] = c[0];   // row mt*16 + g (valid in lanes with t == 0)
        z[mt][1] = c[2];   // row mt*16 + g + 8
    }
}
// Inference forward of the 32 samples in T.X with the hidden activations
// kept in registers: the m16n8 accumulators of n-tiles 2kc and 2kc+1 are,
// after GELU and BF16 rounding, exactly the m16k16 A fragment of k-chunk kc
// of the next layer (rows g, g+8; columns 2t, 2t+1 and 2t+8, 2t+9), so no
// shared-memory round trip is needed.  Same values as mlp_forward.
__device__ __forceinline__ void mlp_logits_regs(const GateWeights &W, const __nv_bfloat16 (*X)[XLD], float z[2][2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        uint32_t a[4];
        load_a<XLD>(X, mt * 16, 0, a);
        float c1[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            uint32_t b[2];
            load_b_wt<XLD>(W.W1, nt * 8, 0, b);
            const float bb0 = W.b1[nt * 8 + 2 * t], bb1 = W.b1[nt * 8 + 2 * t + 1];
            const float c[4] = {bb0, bb1, bb0, bb1};
            mma16816(c1[nt], a, b, c);
        }
        uint32_t h1[2][4];
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
            h1[kc][0] = pack_bf16(gelu(c1[2 * kc][0]), gelu(c1[2 * kc][1]));
            h1[kc][1] = pack_bf16(gelu(c1[2 * kc][2]), gelu(c1[2 * kc][3]));
            h1[kc][2] = pack_bf16(gelu(c1[2 * kc + 1][0]), gelu(c1[2 * kc + 1][1]));
            h1[kc][3] = pack_bf16(gelu(c1[2 * kc + 1][2]), gelu(c1[2 * kc + 1][3]));
        }
        float c2[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const float bb0 = W.b2[nt * 8 + 2 * t], bb1 = W.b2[nt * 8 + 2 * t + 1];
            float c[4] = {bb0, bb1, bb0, bb1};
#pragma unroll
            for (int kc = 0; kc < 2; ++kc) {
                uint32_t b[2];
                load_b_wt<HLD>(W.W2, nt * 8, kc * 16, b);
                float d[4];
                mma16816(d, h1[kc], b, c);
                c[0] = d[0]; c[1] = d[1]; c[2] = d[2]; c[3] = d[3];
            }
            c2[nt][0] = c[0]; c2[nt][1] = c[1]; c2[nt][2] = c[2]; c2[nt][3] = c[3];
        }
        float c[4] = {W.b3, 0.f, W.b3, 0.f};
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
            uint32_t h2[4];
            h2[0] = pack_bf16(gelu(c2[2 * kc][0]), gelu(c2[2 * kc][1]));
            h2[1] = pack_bf16(gelu(c2[2 * kc][2]), gelu(c2[2 * kc][3]));
            h2[2] = pack_bf16(gelu(c2[2 * kc + 1][0]), gelu(c2[2 * kc + 1][1]));
            h2[3] = pack_bf16(gelu(c2[2 * kc + 1][2]), gelu(c2[2 * kc + 1][3]));
            const int k = kc * 16 + 2 * t;
            const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
            const __nv_bfloat16 w0 = g == 0 ? W.w3[k] : zero, w1 = g == 0 ? W.w3[k + 1] : zero;
            const __nv_bfloat16 w8 = g == 0 ? W.w3[k + 8] : zero, w9 = g == 0 ? W.w3[k + 9] : zero;
            uint32_t b[2];
            b[0] = (uint32_t)__bfloat16_as_ushort(w0) | ((uint32_t)__bfloat16_as_ushort(w1) << 16);
            b[1] = (uint32_t)__bfloat16_as_ushort(w8) | ((uint32_t)__bfloat16_as_ushort(w9) << 16);
            float d[4];
            mma16816(d, h2, b, c);
            c[0] = d[0]; c[1] = d[1]; c[2] = d[2]; c[3] = d[3];
        }
        z[mt][0] = c[0];
        z[mt][1] = c[2];
    }
}

// logit of row r (0..31) broadcast to the calling lane
__device__ __forceinline__ float row_logit(const float z[2][2], int r) {
    const int mt = r >> 4, rr = r & 15;
    const int src = (rr & 7) * 4;
    const float v0 = __shfl_sync(0xffffffffu, z[0][0], src), v1 = __shfl_sync(0xffffffffu, z[0][1], src);
    const float v2 = __shfl_sync(0xffffffffu, z[1][0], src), v3 = __shfl_sync(0xffffffffu, z[1][1], src);
    return mt == 0 ? (rr < 8 ? v0 : v1) : (rr < 8 ? v2 : v3);
}

__device__ __forceinline__ void load_weights_smem(GateWeights &W, const float *__restrict__ P) {
    for (int i = threadIdx.x; i < GH * XLD; i += blockDim.x) {
        const int o = i / XLD, k = i % XLD;
        W.W1[o][k] = __float2bfloat16_rn(k < GF ? P[P_W1 + o * GF + k] : 0.f);
    }
    for (int i = threadIdx.x; i < GH * GH; i += blockDim.x) W.W2[i / GH][i % GH] = __float2bfloat16_rn(P[P_W2 + i]);
    for (int i = threadIdx.x; i < GH * (HLD - GH); i += blockDim.x)
        W.W2[i / (HLD - GH)][GH + i % (HLD - GH)] = __float2bfloat16_rn(0.f);
    for (int i = threadIdx.x; i < GH; i += blockDim.x) {
        W.w3[i] = __float2bfloat16_rn(P[P_W3 + i]);
        W.b1[i] = P[P_B1 + i];
        W.b2[i] = P[P_B2 + i];
    }
    if (threadIdx.x == 0) W.b3 = P[P_B3];
}

// ------------------------------------------------------ gate (inference)
// Gate buffers of a handle (int32 / float words): a head of 64 words (the
// current hard-list lengths x, y at 0, 1 and the stage-1 lengths at 2, 3),
// the x hard list (NI + nux entries at most), the y hard list (NI + nuy),
// then per face the stage-1 jump (float; < 0 when the face was hard).
//
// The network runs at RK stage 1 only.  At stages 2 and 3 a face keeps the
// linear path while the largest jump on its stencil stays within
// GUARD_GROWTH x its stage-1 value + GUARD_ABS; a discontinuity moving into
// the stencil during the step (at most one cell at CFL <= 1) fails the test
// and the face takes the full WCNS flux.  Stage-1 hard faces stay on the
// stage-1 list.
constexpr int64_t GATE_LIST_HEAD = 64;
constexpr float GUARD_GROWTH = 1.5f, GUARD_ABS = 1e-3f;

__device__ __forceinline__ void append_hard(bool want, int64_t f, int lane, int32_t *hard, uint32_t *count) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (m) {
        const int leader = __ffs(m) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (want) hard[base + __popc(m & ((1u << lane) - 1u))] = (int32_t)f;
    }
}

// Stage 1: the 32 faces of warp chunk w.  Features, the MLP on the tensor
// cores, and g >= thr: the face gets the linear-weight flux here and its
// jump is kept; otherwise it is appended to the hard list for the full WCNS
// flux.  X columns GF.. of the warp's tile must be zero.  jump_thr >= 0
// replaces the MLP by the plain rule "largest jump <= jump_thr" on the same
// features (the baseline the network is measured against).
template <int DIR>
__device__ __forceinline__ void gate_linear_chunk(const Tables &T, const double4 *__restrict__ cur, double4 *F,
                                                  const GateWeights &W, XTile &Tt, float logit_thr, float jump_thr,
                                                  double lam, double ig1, double g, int32_t *hard, uint32_t *count,
                                                  float *jump1, int64_t w) {
    const int lane = threadIdx.x & 31;
    const int64_t nf = T.NI + (DIR == 0 ? T.nux : T.nuy);
    const int64_t f = w * 32 + lane;
    const bool in = f < nf;
    Prim p0, p1, p2, p3;
    float feat[GF], jm = 0.f;
    if (in) {
        int32_t a, b, c, d;
        face_slots<DIR>(T, f, a, b, c, d);
        p0 = load_prim(cur, a); p1 = load_prim(cur, b); p2 = load_prim(cur, c); p3 = load_prim(cur, d);
        face_features<DIR>(p0, p1, p2, p3, g, feat, &jm);
    } else {
        for (int k = 0; k < GF; ++k) feat[k] = 0.f;
    }
    __syncwarp();
    *reinterpret_cast<uint4 *>(&Tt.X[lane][0]) =
        make_uint4(pack_bf16(feat[0], feat[1]), pack_bf16(feat[2], feat[3]), pack_bf16(feat[4], feat[5]),
                   pack_bf16(feat[6], feat[7]));
    __syncwarp();
    float z[2][2];
    mlp_logits_regs(W, Tt.X, z);
    const float zl = row_logit(z, lane);
    const bool lin = in && (jump_thr >= 0.f ? jm <= jump_thr : zl >= logit_thr);
    if (lin) {
        double out[4];
        face_flux_linear<DIR>(p0, p1, p2, p3, ig1, lam, out);
        F[f] = make_double4(out[0], out[1], out[2], out[3]);
    }
    if (in) jump1[f] = lin ? jm : -1.0f;
    append_hard(in && !lin, f, lane, hard, count);
}

// Stages 2 and 3: the guard on the faces of warp chunk w that were linear
// at stage 1.
template <int DIR>
__device__ __forceinline__ void guard_linear_chunk(const Tables &T, const double4 *__restrict__ cur, double4 *F,
                                                   const float *__restrict__ jump1, double lam, double ig1, double g,
                                                   int32_t *hard, uint32_t *count, int64_t w) {
    const int lane = threadIdx.x & 31;
    const int64_t nf = T.NI + (DIR == 0 ? T.nux : T.nuy);
    const int64_t f = w * 32 + lane;
    const float j1 = f < nf ? jump1[f] : -1.0f;
    bool hardf = false;
    if (j1 >= 0.0f) {
        int32_t a, b, c, d;
        face_slots<DIR>(T, f, a, b, c, d);
        const Prim p0 = load_prim(cur, a), p1 = load_prim(cur, b), p2 = load_prim(cur, c), p3 = load_prim(cur, d);
        if (face_jump<DIR>(p0, p1, p2, p3, g) <= GUARD_GROWTH * j1 + GUARD_ABS) {
            double out[4];
            face_flux_linear<DIR>(p0, p1, p2, p3, ig1, lam, out);
            F[f] = make_double4(out[0], out[1], out[2], out[3]);
        } else {
            hardf = true;
        }
    }
    append_hard(hardf, f, lane, hard, count);
}

// Gate buffer layout of a mesh with faces nfx, nfy.
struct GateLists {
    uint32_t *cnt;      // [0, 1] current hard-list lengths, [2, 3] stage-1 lengths
    int32_t *hx, *hy;   // hard lists
    float *jx, *jy;     // stage-1 jumps
};
__host__ __device__ inline GateLists gate_lists(void *base, int64_t nfx, int64_t nfy) {
    GateLists L;
    int32_t *head = (int32_t *)base;
    L.cnt = (uint32_t *)head;
    L.hx = head + GATE_LIST_HEAD;
    L.hy = L.hx + nfx;
    L.jx = (float *)(L.hy + nfy);
    L.jy = L.jx + nfx;
    return L;
}

}  // namespace fdm
