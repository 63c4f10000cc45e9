// diag.cu — the reference's diagnostic norms on the device.
//
// output_error (src/output_ADT.F90:18-75) compares the density of every
// interior leaf (cell_NS, i.e. key order) with the isentropic vortex of
// strength 5 at (5, 5) and forms L1, L2, Loo over all of them and P1, P2,
// Poo over the refined ones (lvl /= 0), by sequential sums.  Here one kernel
// forms the per-leaf terms in parallel, with the reference's operation
// order, and one warp streams them through shared memory to a single adding
// lane, so the sums are the reference's left-to-right sums.  Only the norms
// (a few doubles) come back to the host.
#include "handle.cuh"

namespace fdm {

constexpr double DIAG_PI = 3.1415926535897932;   // Pi of the reference
constexpr double DIAG_CC1 = 5.0;                 // vortex strength

// per interior leaf: (area, |r|*dx*dy, r*r*dx*dy, |r|); area negated for a
// refined leaf (lvl /= 0)
__global__ void k_error_terms(Tables T, LevelTab LT, const double4 *__restrict__ B0, double g, double4 *terms) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= T.NI) return;
    const int lvl = T.ilvl[i];
    const int32_t s = T.slot_leaf[i];
    const double cx = T.lcx[s], cy = T.lcy[s];
    const double dx = LT.dx[lvl], dy = LT.dy[lvl];
    const double rr = (cx - 5.0) * (cx - 5.0) + (cy - 5.0) * (cy - 5.0);
    const double dT = -(g - 1.0) * (DIAG_CC1 * DIAG_CC1) * exp(1.0 - rr) / (8.0 * g * DIAG_PI * DIAG_PI);
    const double r = B0[i].x - pow(1.0 + dT, 1.0 / (g - 1.0));
    const double area = dx * dy;
    terms[i] = make_double4(lvl != 0 ? -area : area, fabs(r) * dx * dy, r * r * dx * dy, fabs(r));
}

constexpr int DIAG_CHUNK = 512;   // double4 per chunk: 16 KB
__device__ __forceinline__ void cp16_diag(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

// sequential sums in key order; out: uni, l1, l2, loo, patch, p1, p2, poo,
// z, z1, z2, zoo, n_patch, n_0
__global__ void __launch_bounds__(32) k_error_sums(int64_t n, const double4 *__restrict__ terms, double *out) {
    __shared__ double4 buf[2][DIAG_CHUNK];
    const int lane = threadIdx.x;
    const int64_t nch = (n + DIAG_CHUNK - 1) / DIAG_CHUNK;
    auto fetch = [&](int64_t c) {
        const int64_t base = c * DIAG_CHUNK;
        for (int j = lane; j < 2 * DIAG_CHUNK; j += 32) {
            const int64_t e = base + (j >> 1);
            if (e < n) cp16_diag(reinterpret_cast<char *>(&buf[c & 1][j >> 1]) + 16 * (j & 1),
                                 reinterpret_cast<const char *>(terms + e) + 16 * (j & 1));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    double uni = 0.0, l1 = 0.0, l2 = 0.0, loo = 0.0, patch = 0.0, p1 = 0.0, p2 = 0.0, poo = 0.0;
    double z = 0.0, z1 = 0.0, z2 = 0.0, zoo = 0.0;
    long long np = 0, n0 = 0;
    if (nch > 0) fetch(0);
    for (int64_t c = 0; c < nch; ++c) {
        if (c + 1 < nch) {
            fetch(c + 1);
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncwarp();
        if (lane == 0) {
            const int64_t rest = n - c * DIAG_CHUNK;
            const int m = rest < DIAG_CHUNK ? (int)rest : DIAG_CHUNK;
            const double4 *b = buf[c & 1];
            for (int j = 0; j < m; ++j) {
                const double4 t = b[j];
                const double a = fabs(t.x);
                uni = uni + a;
                l1 = l1 + t.y;
                l2 = l2 + t.z;
                loo = fmax(loo, t.w);
                if (t.x < 0.0) {
                    ++np;
                    patch = patch + a;
                    p1 = p1 + t.y;
                    p2 = p2 + t.z;
                    poo = fmax(poo, t.w);
                } else {
                    ++n0;
                    z = z + a;
                    z1 = z1 + t.y;
                    z2 = z2 + t.z;
                    zoo = fmax(zoo, t.w);
                }
            }
        }
        __syncwarp();
    }
    if (lane == 0) {
        const double v[14] = {uni, l1, l2, loo, patch, p1, p2, poo, z, z1, z2, zoo, (double)np, (double)n0};
        for (int k = 0; k < 14; ++k) out[k] = v[k];
    }
}

static inline int nblk_d(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace fdm

using namespace fdm;

// output_error's norms of the current state: norms[0..8] = L1, L2, Loo over
// the interior leaves, P1, P2, Poo over the refined ones, and L1, L2, Loo
// over the level-0 ones; counts[0..2] = interior, level-0 and refined leaves.
extern "C" int fdm_output_error(fdm_handle *h, double *norms, int64_t *counts) {
    if (!h || !norms) return FDM_ERR_ARG;
    if (!h->loaded) { h->err = "no leaf set uploaded"; return FDM_ERR_STATE; }
    DevBuf &d = h->diag;
    FDM_CK(h, d.ensure((size_t)h->NI * 32 + 16 * 8));
    double4 *terms = d.as<double4>();
    double *sums = reinterpret_cast<double *>(terms + h->NI);
    k_error_terms<<<nblk_d(h->NI, 256), 256, 0, h->s>>>(h->tables(), h->lt, h->B[0].as<double4>(), h->G.gama, terms);
    k_error_sums<<<1, 32, 0, h->s>>>(h->NI, terms, sums);
    double s[14];
    FDM_CK(h, cudaMemcpyAsync(s, sums, sizeof s, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    const double uni = s[0], patch = s[4], zz = s[8];
    const long long np = (long long)s[12], n0 = (long long)s[13];
    norms[0] = s[1] / uni;
    norms[1] = sqrt(s[2] / uni);
    norms[2] = s[3];
    norms[3] = np ? s[5] / patch : 0.0;
    norms[4] = np ? sqrt(s[6] / patch) : 0.0;
    norms[5] = s[7];
    norms[6] = n0 ? s[9] / zz : 0.0;
    norms[7] = n0 ? sqrt(s[10] / zz) : 0.0;
    norms[8] = s[11];
    if (counts) {
        counts[0] = h->NI;
        counts[1] = n0;
        counts[2] = np;
    }
    return FDM_OK;
}
