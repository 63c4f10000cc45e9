// diag.cu — the reference's diagnostic norms on the device.
//
// output_error (src/output_ADT.F90:18-75) compares the density of every
// interior leaf (cell_NS, i.e. key order) with the isentropic vortex of
// strength 5 at (5, 5) and forms L1, L2, Loo over all of them and P1, P2,
// Poo over the refined ones (lvl /= 0), by sequential sums.  Here one kernel
// forms the per-leaf terms in parallel, with the reference's operation
// order, and the sums are formed in key order by the exact block-parallel
// summation of ordered_sum.cuh, so they are the reference's left-to-right
// sums.  Only the norms (a few doubles) come back to the host.
#include "handle.cuh"
#include "ordered_sum.cuh"

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

// The sums in key order, each by one block (ordered_sum.cuh), so each is
// the reference's left-to-right sum bit for bit; a sum over the refined
// (or level-0) leaves alone takes +0 for the others.  Block q < 9 forms sum
// q of uni, l1, l2, patch, p1, p2, z, z1, z2; block 9 the maxima (fmax
// ignores order) and the counts.  out: uni, l1, l2, loo, patch, p1, p2,
// poo, z, z1, z2, zoo, n_patch, n_0.
__global__ void __launch_bounds__(OSUM_NT) k_error_sums(int64_t n, const double4 *__restrict__ terms, double *out) {
    __shared__ OSumShared sh;
    __shared__ double red[3][OSUM_NT / 32];
    __shared__ unsigned long long cnt[2];
    const int q = blockIdx.x;
    if (q < 9) {
        const int comp = q % 3;      // area, |r| dx dy, r^2 dx dy
        const int subset = q / 3;    // all, refined, level 0
        const double v = ordered_sum_block<OSUM_NT, OSUM_EPT>(
            [&](int64_t e) {
                const double4 t = terms[e];
                const bool in = subset == 0 || (subset == 1 ? t.x < 0.0 : !(t.x < 0.0));
                const double x = comp == 0 ? fabs(t.x) : (comp == 1 ? t.y : t.z);
                return in ? x : 0.0;
            },
            n, sh);
        const int pos[9] = {0, 1, 2, 4, 5, 6, 8, 9, 10};
        if (threadIdx.x == 0) out[pos[q]] = v;
        return;
    }
    double loo = 0.0, poo = 0.0, zoo = 0.0;
    unsigned long long np = 0, n0 = 0;
    for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
        const double4 t = terms[e];
        loo = fmax(loo, t.w);
        if (t.x < 0.0) { ++np; poo = fmax(poo, t.w); }
        else { ++n0; zoo = fmax(zoo, t.w); }
    }
    for (int d = 16; d > 0; d >>= 1) {
        loo = fmax(loo, __shfl_xor_sync(0xffffffffu, loo, d));
        poo = fmax(poo, __shfl_xor_sync(0xffffffffu, poo, d));
        zoo = fmax(zoo, __shfl_xor_sync(0xffffffffu, zoo, d));
        np += __shfl_xor_sync(0xffffffffu, np, d);
        n0 += __shfl_xor_sync(0xffffffffu, n0, d);
    }
    if (threadIdx.x == 0) { cnt[0] = 0; cnt[1] = 0; }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = loo; red[1][warp] = poo; red[2][warp] = zoo;
        atomicAdd(&cnt[0], np);
        atomicAdd(&cnt[1], n0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            loo = fmax(loo, red[0][w]); poo = fmax(poo, red[1][w]); zoo = fmax(zoo, red[2][w]);
        }
        loo = fmax(loo, red[0][0]); poo = fmax(poo, red[1][0]); zoo = fmax(zoo, red[2][0]);
        out[3] = loo; out[7] = poo; out[11] = zoo;
        out[12] = (double)cnt[0];
        out[13] = (double)cnt[1];
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
    k_error_sums<<<10, OSUM_NT, 0, h->s>>>(h->NI, terms, sums);
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
