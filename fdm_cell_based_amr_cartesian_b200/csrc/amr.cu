// amr.cu — device regrid (src/solution.F90:408-589, src/mesh.F90:199-408).
#include <cub/cub.cuh>

#include "handle.cuh"
#include "topo.cuh"

namespace fdm {

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

void launch_requests(fdm_handle *h, const double4 *cur);

// Urot / Udiv / dux (src/solution.F90:558-589) on the stencil values
// Tip, Tim, Tjp, Tjm of every interior leaf.
__global__ void k_rot_div(Tables T, LevelTab LT, const double4 *__restrict__ B, double *rot, double *div,
                          uint64_t *dfs_key, int32_t *idx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= T.NI) return;
    const int lvl = T.ilvl[i];
    const int32_t *s = T.ist + i * 8;
    const double4 ip = B[s[0]], im = B[s[1]], jp = B[s[2]], jm = B[s[3]];
    const double dy = LT.dy[lvl], dx = LT.dx[lvl], p15 = LT.p15[lvl];
    const double vx = (ip.z - im.z) / (2.0 * dx);
    const double uy = (jp.y - jm.y) / (2.0 * dy);
    rot[i] = fabs(vx - uy) * p15;
    const double ux = (ip.x - im.x) / (2.0 * dx);
    const double vy = (jp.x - jm.x) / (2.0 * dy);
    div[i] = (fabs(ux) + fabs(vy)) * p15;
    // traversal order of solute_div_rot: roots row-major, sons 1,2,3,4
    const uint64_t key = T.lkey[T.slot_leaf[i]];
    const uint64_t path = key_pos(key) & ((1ull << 30) - 1ull);
    dfs_key[i] = ((key >> 34) << 30) | (path ^ ((path & 0x2AAAAAAAull) >> 1));
    idx[i] = (int32_t)i;
}

// Srot = Srot + rot**2 ... in traversal order: one thread, the sum is a
// sequence of roundings that no parallel order reproduces
__global__ void k_ordered_sums(int64_t NI, const int32_t *order, const double *rot, const double *div,
                               double *out) {
    if (threadIdx.x || blockIdx.x) return;
    double sr = 0.0, sd = 0.0;
    for (int64_t k = 0; k < NI; ++k) {
        const int32_t i = order[k];
        sr = sr + rot[i] * rot[i];
        sd = sd + div[i] * div[i];
    }
    out[0] = sr;
    out[1] = sd;
    out[2] = (double)NI;
}

// rot/div of the current state into rot/div buffers; ordered sums to out3
static int compute_rot_div(fdm_handle *h, double *rot, double *div, double *out3) {
    const int64_t NI = h->NI;
    launch_requests(h, h->B[0].as<double4>());
    Carve cv;
    cv.add(NI * 8); cv.add(NI * 8); cv.add(NI * 4); cv.add(NI * 4);
    FDM_CK(h, h->tmp[0].ensure(cv.total));
    uint64_t *k0 = cv.at<uint64_t>(h->tmp[0], 0), *k1 = cv.at<uint64_t>(h->tmp[0], 1);
    int32_t *i0 = cv.at<int32_t>(h->tmp[0], 2), *i1 = cv.at<int32_t>(h->tmp[0], 3);
    k_rot_div<<<nblk(NI, 256), 256, 0, h->s>>>(h->tables(), h->lt, h->B[0].as<double4>(), rot, div, k0, i0);
    size_t bytes = 0;
    FDM_CK(h, cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0, k1, i0, i1, (int)NI, 0, 64, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceRadixSort::SortPairs(h->cub_tmp.p, bytes, k0, k1, i0, i1, (int)NI, 0, 64, h->s));
    k_ordered_sums<<<1, 32, 0, h->s>>>(NI, i1, rot, div, out3);
    return FDM_OK;
}

int run_amr(fdm_handle *h) {
    h->err = "device regrid not built yet";
    return FDM_ERR_UNSUPPORTED;
}

}  // namespace fdm

extern "C" int fdm_debug_rot_div(fdm_handle *h, int64_t cap, double *rot, double *div, double *sums) {
    using namespace fdm;
    if (!h) return FDM_ERR_ARG;
    if (!h->loaded) return FDM_ERR_STATE;
    if (cap < h->NI) return arg_fail(h, "capacity below the interior leaf count");
    DevBuf d;
    Carve cv;
    cv.add(h->NI * 8); cv.add(h->NI * 8); cv.add(3 * 8);
    FDM_CK(h, d.ensure(cv.total));
    double *dr = cv.at<double>(d, 0), *dd = cv.at<double>(d, 1), *ds = cv.at<double>(d, 2);
    int rc = compute_rot_div(h, dr, dd, ds);
    if (rc) return rc;
    if (rot) FDM_CK(h, cudaMemcpyAsync(rot, dr, h->NI * 8, cudaMemcpyDeviceToHost, h->s));
    if (div) FDM_CK(h, cudaMemcpyAsync(div, dd, h->NI * 8, cudaMemcpyDeviceToHost, h->s));
    if (sums) FDM_CK(h, cudaMemcpyAsync(sums, ds, 24, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    d.release();
    return FDM_OK;
}
