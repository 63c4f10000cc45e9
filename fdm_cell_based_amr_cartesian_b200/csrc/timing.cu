// timing.cu — CUDA-event timing of the stage kernels on the handle's stream
// and a DFMA throughput probe (the FP64 roofline denominator).
#include "handle.cuh"

namespace fdm {

// 8 independent DFMA chains per thread; 2 flops per DFMA
__global__ void k_dfma(double *out, int iters, double a, double b) {
    double x0 = threadIdx.x * 1e-3, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678) out[0] = s;   // keeps the chains live
}

}  // namespace fdm

using namespace fdm;

extern "C" int fdm_time_kernels(fdm_handle *h, int32_t reps, double *ms) {
    if (!h || !ms || reps <= 0) return FDM_ERR_ARG;
    if (!h->loaded) return FDM_ERR_STATE;
    cudaEvent_t e[2];
    FDM_CK(h, cudaEventCreate(&e[0]));
    FDM_CK(h, cudaEventCreate(&e[1]));
    double4 *b0 = h->B[0].as<double4>(), *b1 = h->B[1].as<double4>();
    for (int which = 0; which < 4; ++which) {
        // one untimed launch, then reps timed launches
        for (int r = 0; r <= reps; ++r) {
            if (r == 1) FDM_CK(h, cudaEventRecord(e[0], h->s));
            if (which == 0) launch_faces(h, b0, 1 + r % 3);   // gated: stage-1 and stage-2/3 kinds in turn
            else if (which == 1) launch_cells(h, b0, b0, b1, 2, 0);
            else if (which == 2) launch_requests(h, b0);
            else launch_ghosts(h, b1, 3);
        }
        FDM_CK(h, cudaEventRecord(e[1], h->s));
        FDM_CK(h, cudaEventSynchronize(e[1]));
        float t = 0.f;
        FDM_CK(h, cudaEventElapsedTime(&t, e[0], e[1]));
        ms[which] = (double)t / reps;
    }
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
    return FDM_OK;
}

namespace fdm {
const char *face_variant_name(int v);
constexpr int N_FACE_VARIANTS = FDM_FACE_VARIANTS;
}

// Autotuner: times every launch shape of the face kernel on the current leaf
// set (CUDA events on the handle's stream, reps launches each, after one
// untimed launch) and keeps the fastest.  ms[v] receives the average ms per
// (x + y) launch pair of variant v.
extern "C" int fdm_autotune(fdm_handle *h, int32_t reps, int32_t *best, double *ms) {
    if (!h || reps <= 0) return FDM_ERR_ARG;
    if (!h->loaded) return FDM_ERR_STATE;
    cudaEvent_t e[2];
    FDM_CK(h, cudaEventCreate(&e[0]));
    FDM_CK(h, cudaEventCreate(&e[1]));
    const int keep = h->face_variant;
    double bt = 1e30;
    int bv = keep;
    for (int v = 0; v < N_FACE_VARIANTS; ++v) {
        h->face_variant = v;
        launch_faces(h, h->B[0].as<double4>(), 1);
        FDM_CK(h, cudaEventRecord(e[0], h->s));
        for (int r = 0; r < reps; ++r) launch_faces(h, h->B[0].as<double4>(), 1);
        FDM_CK(h, cudaEventRecord(e[1], h->s));
        FDM_CK(h, cudaEventSynchronize(e[1]));
        float t = 0.f;
        FDM_CK(h, cudaEventElapsedTime(&t, e[0], e[1]));
        const double avg = (double)t / reps;
        if (ms) ms[v] = avg;
        if (avg < bt) { bt = avg; bv = v; }
    }
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
    h->face_variant = bv;
    h->graph_version = -1;   // the step graph holds the old launch shape
    if (best) *best = bv;
    return FDM_OK;
}

namespace fdm {
int count_nr_fallbacks(fdm_handle *h, int64_t out[2]);
}
// x and y faces whose branch-free division falls back to the compiler's on
// the current state (face variants 7-10, 13, 14)
extern "C" int fdm_debug_nr_fallbacks(fdm_handle *h, int64_t *out) {
    if (!h || !out) return FDM_ERR_ARG;
    if (!h->loaded) return FDM_ERR_STATE;
    return fdm::count_nr_fallbacks(h, out);
}

extern "C" int fdm_set_variant(fdm_handle *h, int32_t face_variant) {
    if (!h || face_variant < 0 || face_variant >= N_FACE_VARIANTS) return FDM_ERR_ARG;
    h->face_variant = face_variant;
    h->graph_version = -1;
    return FDM_OK;
}

extern "C" int fdm_fp64_peak(double *tflops) {
    if (!tflops) return FDM_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FDM_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    double *out = nullptr;
    if (cudaMalloc(&out, 8) != cudaSuccess) return FDM_ERR_CUDA;
    const int threads = 256, blocks = sms * 8, iters = 1 << 14;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_dfma<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(a);
    const int reps = 5;
    for (int r = 0; r < reps; ++r) k_dfma<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * (double)iters * threads * blocks * reps;
    *tflops = flops / (t * 1e-3) / 1e12;
    return cudaGetLastError() == cudaSuccess ? FDM_OK : FDM_ERR_CUDA;
}
