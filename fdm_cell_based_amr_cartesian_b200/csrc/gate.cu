// gate.cu — learned smoothness gate of the face flux.
//
// A small MLP (8 -> 32 -> 32 -> 1, GELU, sigmoid; BF16 weights and
// activations, FP32 accumulation on the tensor cores through
// mma.sync.m16n8k16) decides per face whether the linear WCNS weights
// suffice.  On such faces the flux is the component-wise linear
// reconstruction of the conserved variables and fluxes (no characteristic
// projection, no nonlinear weights); everywhere else the plain scheme of
// numerics.cuh runs unchanged.  No reference counterpart: the reference
// always evaluates the nonlinear weights (src/nnd_center_RK.F90:310-353).
//
// The same file holds the training side: per-face (features, target)
// samples emitted by the plain solver, a fused forward+backward kernel that
// accumulates the gradients of a minibatch, and Adam.
#include <algorithm>

#include "gate_items.cuh"

namespace fdm {

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

// Stage 1, persistent: each warp takes 32 faces at a time.
template <int DIR>
__global__ void __launch_bounds__(128, 4) k_gate_linear(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                        const float *__restrict__ P, float logit_thr,
                                                        float jump_thr, const DevScalars *__restrict__ sc, double g,
                                                        int32_t *hard,
                                                        uint32_t *count, float *jump1) {
    __shared__ GateWeights W;
    __shared__ XTile tiles[4];
    load_weights_smem(W, P);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t nf = T.NI + (DIR == 0 ? T.nux : T.nuy);
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    const double ig1 = 1.0 / (g - 1.0);
    XTile &Tt = tiles[wid];
    for (int k = GF; k < XLD; ++k) Tt.X[lane][k] = __float2bfloat16_rn(0.f);
    const int64_t nwarps = (int64_t)gridDim.x * 4;
    for (int64_t w = blockIdx.x * 4 + wid; w * 32 < nf; w += nwarps)
        gate_linear_chunk<DIR>(T, cur, F, W, Tt, logit_thr, jump_thr, lam, ig1, g, hard, count, jump1, w);
}

// Stages 2 and 3: the guard on the faces that were linear at stage 1.
template <int DIR>
__global__ void __launch_bounds__(256) k_guard_linear(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                      const float *__restrict__ jump1,
                                                      const DevScalars *__restrict__ sc, double g, int32_t *hard,
                                                      uint32_t *count) {
    const int64_t nf = T.NI + (DIR == 0 ? T.nux : T.nuy);
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    const double ig1 = 1.0 / (g - 1.0);
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t w = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < nf; w += nwarps)
        guard_linear_chunk<DIR>(T, cur, F, jump1, lam, ig1, g, hard, count, w);
}

// full WCNS flux of the faces on the hard list
template <int DIR>
__global__ void __launch_bounds__(256, 2) k_faces_list(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                       const int32_t *__restrict__ hard,
                                                       const uint32_t *__restrict__ count,
                                                       const DevScalars *__restrict__ sc, double g) {
    const int64_t n = *count;
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        face_item<DIR>(T, cur, F, lam, g, hard[i]);
}

// --------------------------------------------------- training samples
// (features, target) of every stride-th face of the current state; target
// = exp(-dev/tau) with dev the largest nonlinear-weight deviation.
template <int DIR>
__global__ void k_face_samples(Tables T, const double4 *__restrict__ cur, double gama, int64_t stride, int64_t phase,
                               double tau, float *feat, float *target, int64_t out0, int64_t cap) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nf = T.NI + (DIR == 0 ? T.nux : T.nuy);
    const int64_t f = j * stride + phase;
    if (f >= nf) return;
    const int64_t o = out0 + j;
    if (o >= cap) return;
    int32_t a, b, c, d;
    face_slots<DIR>(T, f, a, b, c, d);
    const Prim p0 = load_prim(cur, a), p1 = load_prim(cur, b), p2 = load_prim(cur, c), p3 = load_prim(cur, d);
    float fv[GF];
    face_features<DIR>(p0, p1, p2, p3, gama, fv);
    for (int k = 0; k < GF; ++k) feat[o * GF + k] = fv[k];
    target[o] = (float)exp(-face_weight_deviation<DIR>(p0, p1, p2, p3, gama) / tau);
}

// ----------------------------------------------------------- training
// Fused forward + backward of the weighted cross entropy
// -(y log g + neg_w (1-y) log(1-g)), g = sigmoid(z), for a minibatch; gradients
// of the mean loss accumulate into grad (FP32 atomics), the loss sum into
// loss.  Samples idx0 + k*step (mod n), k < B.
struct TrainTile {
    WarpTile t;
    __nv_bfloat16 DA2[32][HLD], DA1[32][HLD];
    float dz[32];
};
__global__ void __launch_bounds__(64) k_mlp_grad(const float *__restrict__ X, const float *__restrict__ Y, int64_t n,
                                                 int64_t idx0, int64_t step, int64_t B, const float *__restrict__ P,
                                                 float neg_w, float *grad, float *loss) {
    __shared__ GateWeights W;
    __shared__ TrainTile tiles[2];
    load_weights_smem(W, P);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    TrainTile &Tt = tiles[wid];
    // per-warp gradient accumulators
    float gW2[2][4][4], gW1[2][4];   // dW2: [mt over out][nt over in][i]; dW1: [mt over out][i], n = features
    for (int a = 0; a < 2; ++a) {
        for (int b = 0; b < 4; ++b) for (int i = 0; i < 4; ++i) gW2[a][b][i] = 0.f;
        for (int i = 0; i < 4; ++i) gW1[a][i] = 0.f;
    }
    float gb1 = 0.f, gb2 = 0.f, gw3 = 0.f, gb3 = 0.f, ls = 0.f;   // lane j holds index j
    const float invB = 1.0f / (float)B;
    const int64_t ngroups = (B + 31) / 32;
    for (int64_t grp = blockIdx.x * 2 + wid; grp < ngroups; grp += (int64_t)gridDim.x * 2) {
        const int64_t k = grp * 32 + lane;
        const bool valid = k < B;
        const int64_t s = (idx0 + k * step) % n;
        float y = 0.f;
        for (int q = 0; q < XLD; ++q) Tt.t.X[lane][q] = __float2bfloat16_rn(valid && q < GF ? X[s * GF + q] : 0.f);
        if (valid) y = Y[s];
        __syncwarp();
        float a1[2][4][4], a2[2][4][4], z[2][2];
        mlp_forward(W, Tt.t, a1, a2, z);
        const float zl = row_logit(z, lane);
        const float gs = 1.0f / (1.0f + expf(-zl));
        if (valid) {
            const float e = 1e-7f;
            ls += -(y * logf(gs + e) + neg_w * (1.0f - y) * logf(1.0f - gs + e));
        }
        // d/dz of -(y log g + a (1-y) log(1-g)) = g (y + a (1-y)) - y
        Tt.dz[lane] = valid ? (gs * (y + neg_w * (1.0f - y)) - y) * invB : 0.f;
        __syncwarp();
        // dh2 = dz w3, da2 = dh2 gelu'(a2)
        for (int mt = 0; mt < 2; ++mt)
            for (int nt = 0; nt < 4; ++nt)
                for (int i = 0; i < 4; ++i) {
                    const int r = mt * 16 + g + 8 * (i >> 1), c = nt * 8 + 2 * t + (i & 1);
                    const float v = Tt.dz[r] * __bfloat162float(W.w3[c]) * gelu_grad(a2[mt][nt][i]);
                    Tt.DA2[r][c] = __float2bfloat16_rn(v);
                }
        __syncwarp();
        // dw3[j] = sum_s h2[s][j] dz[s]; db3 = sum dz; db2[j] = sum_s da2[s][j]
        {
            float sw = 0.f, sb = 0.f;
            for (int r = 0; r < 32; ++r) {
                sw += __bfloat162float(Tt.t.H2[r][lane]) * Tt.dz[r];
            }
            gw3 += sw;
            for (int r = 0; r < 32; ++r) sb += __bfloat162float(Tt.DA2[r][lane]);
            gb2 += sb;
            gb3 += Tt.dz[lane];
        }
        // dh1 = DA2 W2 (B[k=o][n=i] = W2[o][i]); da1 = dh1 gelu'(a1)
        for (int mt = 0; mt < 2; ++mt)
            for (int nt = 0; nt < 4; ++nt) {
                float c[4] = {0.f, 0.f, 0.f, 0.f};
                for (int kc = 0; kc < 2; ++kc) {
                    uint32_t a[4], b[2];
                    load_a<HLD>(Tt.DA2, mt * 16, kc * 16, a);
                    const int nn = nt * 8 + g, kk = kc * 16 + 2 * t;
                    b[0] = (uint32_t)__bfloat16_as_ushort(W.W2[kk][nn]) | ((uint32_t)__bfloat16_as_ushort(W.W2[kk + 1][nn]) << 16);
                    b[1] = (uint32_t)__bfloat16_as_ushort(W.W2[kk + 8][nn]) | ((uint32_t)__bfloat16_as_ushort(W.W2[kk + 9][nn]) << 16);
                    float d[4];
                    mma16816(d, a, b, c);
                    c[0] = d[0]; c[1] = d[1]; c[2] = d[2]; c[3] = d[3];
                }
                for (int i = 0; i < 4; ++i) {
                    const int r = mt * 16 + g + 8 * (i >> 1), cc = nt * 8 + 2 * t + (i & 1);
                    Tt.DA1[r][cc] = __float2bfloat16_rn(c[i] * gelu_grad(a1[mt][nt][i]));
                }
            }
        __syncwarp();
        {
            float sb = 0.f;
            for (int r = 0; r < 32; ++r) sb += __bfloat162float(Tt.DA1[r][lane]);
            gb1 += sb;
        }
        // dW2[o][i] += sum_s DA2[s][o] H1[s][i]: A[m=o][k=s], B[k=s][n=i]
        for (int mt = 0; mt < 2; ++mt)
            for (int kc = 0; kc < 2; ++kc) {
                uint32_t a[4];
                {
                    const int o0 = mt * 16 + g, o1 = o0 + 8, s0 = kc * 16 + 2 * t, s1 = s0 + 8;
                    a[0] = (uint32_t)__bfloat16_as_ushort(Tt.DA2[s0][o0]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA2[s0 + 1][o0]) << 16);
                    a[1] = (uint32_t)__bfloat16_as_ushort(Tt.DA2[s0][o1]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA2[s0 + 1][o1]) << 16);
                    a[2] = (uint32_t)__bfloat16_as_ushort(Tt.DA2[s1][o0]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA2[s1 + 1][o0]) << 16);
                    a[3] = (uint32_t)__bfloat16_as_ushort(Tt.DA2[s1][o1]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA2[s1 + 1][o1]) << 16);
                }
                for (int nt = 0; nt < 4; ++nt) {
                    uint32_t b[2];
                    const int nn = nt * 8 + g, kk = kc * 16 + 2 * t;
                    b[0] = (uint32_t)__bfloat16_as_ushort(Tt.t.H1[kk][nn]) | ((uint32_t)__bfloat16_as_ushort(Tt.t.H1[kk + 1][nn]) << 16);
                    b[1] = (uint32_t)__bfloat16_as_ushort(Tt.t.H1[kk + 8][nn]) | ((uint32_t)__bfloat16_as_ushort(Tt.t.H1[kk + 9][nn]) << 16);
                    float d[4];
                    mma16816(d, a, b, gW2[mt][nt]);
                    for (int i = 0; i < 4; ++i) gW2[mt][nt][i] = d[i];
                }
            }
        // dW1[o][f] += sum_s DA1[s][o] X[s][f]: N = 8 features (one n-tile)
        for (int mt = 0; mt < 2; ++mt)
            for (int kc = 0; kc < 2; ++kc) {
                uint32_t a[4], b[2];
                const int o0 = mt * 16 + g, o1 = o0 + 8, s0 = kc * 16 + 2 * t, s1 = s0 + 8;
                a[0] = (uint32_t)__bfloat16_as_ushort(Tt.DA1[s0][o0]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA1[s0 + 1][o0]) << 16);
                a[1] = (uint32_t)__bfloat16_as_ushort(Tt.DA1[s0][o1]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA1[s0 + 1][o1]) << 16);
                a[2] = (uint32_t)__bfloat16_as_ushort(Tt.DA1[s1][o0]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA1[s1 + 1][o0]) << 16);
                a[3] = (uint32_t)__bfloat16_as_ushort(Tt.DA1[s1][o1]) | ((uint32_t)__bfloat16_as_ushort(Tt.DA1[s1 + 1][o1]) << 16);
                const int kk = kc * 16 + 2 * t;
                b[0] = (uint32_t)__bfloat16_as_ushort(Tt.t.X[kk][g]) | ((uint32_t)__bfloat16_as_ushort(Tt.t.X[kk + 1][g]) << 16);
                b[1] = (uint32_t)__bfloat16_as_ushort(Tt.t.X[kk + 8][g]) | ((uint32_t)__bfloat16_as_ushort(Tt.t.X[kk + 9][g]) << 16);
                float d[4];
                mma16816(d, a, b, gW1[mt]);
                for (int i = 0; i < 4; ++i) gW1[mt][i] = d[i];
            }
        __syncwarp();
    }
    // flush the warp's accumulators
    for (int mt = 0; mt < 2; ++mt) {
        for (int nt = 0; nt < 4; ++nt)
            for (int i = 0; i < 4; ++i) {
                const int o = mt * 16 + g + 8 * (i >> 1), in = nt * 8 + 2 * t + (i & 1);
                atomicAdd(grad + P_W2 + o * GH + in, gW2[mt][nt][i]);
            }
        for (int i = 0; i < 4; ++i) {
            const int o = mt * 16 + g + 8 * (i >> 1), fi = 2 * t + (i & 1);
            atomicAdd(grad + P_W1 + o * GF + fi, gW1[mt][i]);
        }
    }
    atomicAdd(grad + P_B1 + lane, gb1);
    atomicAdd(grad + P_B2 + lane, gb2);
    atomicAdd(grad + P_W3 + lane, gw3);
    for (int o = 16; o; o >>= 1) {
        gb3 += __shfl_xor_sync(0xffffffffu, gb3, o);
        ls += __shfl_xor_sync(0xffffffffu, ls, o);
    }
    if (lane == 0) {
        atomicAdd(grad + P_B3, gb3);
        atomicAdd(loss, ls);
    }
}

// Adam (FP32 master weights)
__global__ void k_adam(float *P, const float *grad, float *m, float *v, int64_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// gate probabilities of given feature rows (evaluation / tests)
__global__ void __launch_bounds__(128) k_mlp_eval(const float *__restrict__ X, int64_t n, const float *__restrict__ P,
                                                  float *prob) {
    __shared__ GateWeights W;
    __shared__ XTile tiles[4];
    load_weights_smem(W, P);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t r = (blockIdx.x * 4 + wid) * 32 + lane;
    XTile &Tt = tiles[wid];
    for (int q = 0; q < XLD; ++q) Tt.X[lane][q] = __float2bfloat16_rn(r < n && q < GF ? X[r * GF + q] : 0.f);
    __syncwarp();
    float z[2][2];
    mlp_logits_regs(W, Tt.X, z);
    const float zl = row_logit(z, lane);
    if (r < n) prob[r] = 1.0f / (1.0f + expf(-zl));
}

// ------------------------------------------------------ gated face flux
static int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

void launch_gated_faces(fdm_handle *h, const double4 *cur, int krk) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    const int64_t nfx = h->NI + h->nux, nfy = h->NI + h->nuy;
    const GateLists GL = gate_lists(h->gate_flag.p, nfx, nfy);
    uint32_t *cnt = GL.cnt;
    int32_t *hx = GL.hx, *hy = GL.hy;
    float *jx = GL.jx, *jy = GL.jy;
    const float *P = h->gate_params.as<float>();
    const int sms = sm_count();
    const int lx = (int)std::min<int64_t>(nblk(nfx, 256), 2 * sms), ly = (int)std::min<int64_t>(nblk(nfy, 256), 2 * sms);
    if (krk == 1 || !h->gate_stage1_valid) {
        const int gx = (int)std::min<int64_t>(nblk(nfx, 128), 4 * sms), gy = (int)std::min<int64_t>(nblk(nfy, 128), 4 * sms);
        cudaMemsetAsync(cnt, 0, 2 * sizeof(uint32_t), h->s);
        if (gx > 0) k_gate_linear<0><<<gx, 128, 0, h->s>>>(T, cur, h->Fx.as<double4>(), P, h->gate_logit_thr, h->gate_jump_thr, sc, h->G.gama, hx, cnt, jx);
        if (gy > 0) k_gate_linear<1><<<gy, 128, 0, h->s>>>(T, cur, h->Fy.as<double4>(), P, h->gate_logit_thr, h->gate_jump_thr, sc, h->G.gama, hy, cnt + 1, jy);
        cudaMemcpyAsync(cnt + 2, cnt, 2 * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->s);
        h->gate_stage1_valid = true;
    } else {
        const int gx = (int)std::min<int64_t>(nblk(nfx, 256), 4 * sms), gy = (int)std::min<int64_t>(nblk(nfy, 256), 4 * sms);
        cudaMemcpyAsync(cnt, cnt + 2, 2 * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->s);
        if (gx > 0) k_guard_linear<0><<<gx, 256, 0, h->s>>>(T, cur, h->Fx.as<double4>(), jx, sc, h->G.gama, hx, cnt);
        if (gy > 0) k_guard_linear<1><<<gy, 256, 0, h->s>>>(T, cur, h->Fy.as<double4>(), jy, sc, h->G.gama, hy, cnt + 1);
    }
    if (h->p.flux_variant == 1) {
        launch_faces_list_fast(h, cur, hx, hy, cnt, lx, ly);
        return;
    }
    if (lx > 0) k_faces_list<0><<<lx, 256, 0, h->s>>>(T, cur, h->Fx.as<double4>(), hx, cnt, sc, h->G.gama);
    if (ly > 0) k_faces_list<1><<<ly, 256, 0, h->s>>>(T, cur, h->Fy.as<double4>(), hy, cnt + 1, sc, h->G.gama);
}

size_t gate_list_bytes(const fdm_handle *h) {
    return (size_t)(GATE_LIST_HEAD + 2 * (2 * h->NI + h->nux + h->nuy)) * sizeof(int32_t);
}

}  // namespace fdm

using namespace fdm;

extern "C" int fdm_gate_param_count(void) { return P_N; }

// faces that took the linear path in the last gated stage, and all faces
extern "C" int fdm_gate_stats(fdm_handle *h, int64_t *gated, int64_t *total) {
    if (!h) return FDM_ERR_ARG;
    if (!h->loaded) return FDM_ERR_STATE;
    const int64_t n = 2 * h->NI + h->nux + h->nuy;
    if (total) *total = n;
    if (!gated) return FDM_OK;
    if (!h->gate_on) { *gated = 0; return FDM_OK; }
    uint32_t c[2] = {0, 0};
    cudaMemcpyAsync(c, h->gate_flag.p, sizeof c, cudaMemcpyDeviceToHost, h->s);
    const cudaError_t e = cudaStreamSynchronize(h->s);
    if (e != cudaSuccess) return cuda_fail(h, e, "fdm_gate_stats");
    *gated = n - (int64_t)c[0] - (int64_t)c[1];
    return FDM_OK;
}

extern "C" int fdm_gate_set(fdm_handle *h, const float *params, float threshold, int32_t enable) {
    if (!h) return FDM_ERR_ARG;
    if (enable) {
        if (!params || !(threshold > 0.f && threshold < 1.f)) return FDM_ERR_ARG;
        FDM_CK(h, h->gate_params.ensure(P_N * sizeof(float)));
        FDM_CK(h, cudaMemcpy(h->gate_params.p, params, P_N * sizeof(float), cudaMemcpyHostToDevice));
        h->gate_logit_thr = logf(threshold / (1.f - threshold));
        h->gate_jump_thr = -1.f;
    }
    h->gate_on = enable != 0;
    h->gate_stage1_valid = false;
    h->graph_version = -1;
    return FDM_OK;
}

// The plain jump rule in place of the network: a face is linear at stage 1
// when its largest normalised jump (the unsquashed gate features) is at most
// jump_threshold; a negative value restores the network.  The gate must have
// been enabled by fdm_gate_set.
extern "C" int fdm_gate_set_jump_rule(fdm_handle *h, float jump_threshold) {
    if (!h) return FDM_ERR_ARG;
    if (!h->gate_on || !h->gate_params.p) { h->err = "the gate is off: fdm_gate_set first"; return FDM_ERR_STATE; }
    h->gate_jump_thr = jump_threshold >= 0.f ? jump_threshold : -1.f;
    h->gate_stage1_valid = false;
    h->graph_version = -1;
    return FDM_OK;
}

extern "C" int fdm_gate_samples(fdm_handle *h, int64_t stride, int64_t phase, double tau, float *feat_dev,
                                float *target_dev, int64_t offset, int64_t cap, int64_t *n_written) {
    if (!h || stride <= 0 || phase < 0 || phase >= stride || !(tau > 0) || !feat_dev || !target_dev) return FDM_ERR_ARG;
    if (!h->loaded) return FDM_ERR_STATE;
    const Tables T = h->tables();
    const int64_t nfx = h->NI + h->nux, nfy = h->NI + h->nuy;
    const int64_t jx = (nfx - phase + stride - 1) / stride, jy = (nfy - phase + stride - 1) / stride;
    const double4 *cur = h->B[0].as<double4>();
    launch_requests(h, cur);
    if (jx > 0)
        k_face_samples<0><<<nblk(jx, 128), 128, 0, h->s>>>(T, cur, h->G.gama, stride, phase, tau, feat_dev,
                                                            target_dev, offset, cap);
    if (jy > 0)
        k_face_samples<1><<<nblk(jy, 128), 128, 0, h->s>>>(T, cur, h->G.gama, stride, phase, tau, feat_dev,
                                                            target_dev, offset + jx, cap);
    FDM_CK(h, cudaStreamSynchronize(h->s));
    int64_t w = jx + jy;
    if (offset + w > cap) w = cap > offset ? cap - offset : 0;
    if (n_written) *n_written = w;
    return FDM_OK;
}

// One Adam step on a minibatch of B samples (idx0 + k*step mod n).
extern "C" int fdm_gate_train_step(const float *X, const float *Y, int64_t n, int64_t idx0, int64_t step, int64_t B,
                                   float neg_weight, float *params, float *grad, float *adam_m, float *adam_v,
                                   int64_t t, float lr, float *loss, void *stream) {
    if (!X || !Y || n <= 0 || B <= 0 || !params || !grad || !adam_m || !adam_v || !loss || t <= 0 ||
        !(neg_weight > 0.f))
        return FDM_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(grad, 0, P_N * sizeof(float), s) != cudaSuccess) return FDM_ERR_CUDA;
    if (cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) return FDM_ERR_CUDA;
    const int64_t ngroups = (B + 31) / 32;
    int blocks = (int)((ngroups + 1) / 2);
    if (blocks > 1184) blocks = 1184;
    k_mlp_grad<<<blocks, 64, 0, s>>>(X, Y, n, idx0, step, B, params, neg_weight, grad, loss);
    if (lr > 0.f) {
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
        k_adam<<<(P_N + 255) / 256, 256, 0, s>>>(params, grad, adam_m, adam_v, P_N, lr, b1, b2, 1e-8f, c1, c2);
    }
    return cudaGetLastError() == cudaSuccess ? FDM_OK : FDM_ERR_CUDA;
}

extern "C" int fdm_gate_eval(const float *X, int64_t n, const float *params, float *prob, void *stream) {
    if (!X || n <= 0 || !params || !prob) return FDM_ERR_ARG;
    k_mlp_eval<<<(int)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(X, n, params, prob);
    return cudaGetLastError() == cudaSuccess ? FDM_OK : FDM_ERR_CUDA;
}
