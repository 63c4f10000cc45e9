// static_uniform.cu — one SSP-RK3 step of the WCNS scheme on a uniform
// periodic grid without any device allocation.
//
// Some callers cannot allocate device memory: a Fortran or C host whose GPU
// memory is handed out by its own pool (an OpenACC or CUDA Fortran runtime
// that owns the heap), code that must run under a fixed memory budget set
// at start-up, or a process that forbids cudaMalloc after initialisation.
// For them this entry point keeps its working memory (the two intermediate
// stage states and the x/y face fluxes) in one file-scope static __device__
// array of fixed size (8.5 MiB), which every GPU that loads libfdm holds
// until the process exits.  The caller passes the input and output states.
//
// The arithmetic is the exact build's (same face_flux and update as the
// handle path, same operation order), so the result equals fdm_time_advance_rk
// on the same uniform periodic leaf set.
#include <algorithm>
#include <cstdint>

#include "handle.cuh"
#include "numerics.cuh"

namespace fdm {
namespace uniform_static {

// worst cases over 3 <= nx, ny <= FDM_STATIC_MAX_SIDE, nx*ny <= FDM_STATIC_MAX_CELLS
constexpr int64_t GRID_CAP = 72100;   // (nx+6)*(ny+6) records
constexpr int64_t FACE_CAP = 66560;   // max((nx+1)*ny, nx*(ny+1)) records
constexpr int64_t SCRATCH_RECORDS = 2 * GRID_CAP + 2 * FACE_CAP;

// The scratch.  In host code this name is only a stand-in for the device
// symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double4 scratch[SCRATCH_RECORDS];

// Device address of the scratch on the current device.  It is looked up on
// every call, with the caller's device current: a cached address would go
// stale when the context that loaded the module is torn down and created
// again (cudaDeviceReset), and the lookup is a cheap runtime call.  The
// first call on a device also loads the module there (lazy loading).
static cudaError_t scratch_address(double4 **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, scratch);
    if (e != cudaSuccess) return e;
    *out = (double4 *)p;
    return cudaSuccess;
}

struct Grid2 {
    int nx, ny, W;   // W = nx + 6 records per row
    __device__ __forceinline__ int64_t at(int r, int c) const { return (int64_t)r * W + c; }
};

// face i of row r in x lies between interior columns 3+i-1 and 3+i
template <int DIR>
__global__ void __launch_bounds__(128) k_ufaces(Grid2 G, const double4 *__restrict__ cur, double4 *F,
                                                double g, double lam) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int nfr = DIR == 0 ? G.nx + 1 : G.nx;          // faces per row
    const int nrow = DIR == 0 ? G.ny : G.ny + 1;
    if (t >= (int64_t)nfr * nrow) return;
    const int r = (int)(t / nfr), i = (int)(t % nfr);
    int64_t a, b, c, d;
    if (DIR == 0) {
        const int row = 3 + r, col = 3 + i;
        a = G.at(row, col - 2); b = G.at(row, col - 1); c = G.at(row, col); d = G.at(row, col + 1);
    } else {
        const int row = 3 + r, col = 3 + i;
        a = G.at(row - 2, col); b = G.at(row - 1, col); c = G.at(row, col); d = G.at(row + 1, col);
    }
    double out[4];
    face_flux<DIR>(load_prim(cur, a), load_prim(cur, b), load_prim(cur, c), load_prim(cur, d), g, lam, out);
    F[t] = make_double4(out[0], out[1], out[2], out[3]);
}

// LXL + updateRK for every interior cell (same operations as k_cells)
__global__ void __launch_bounds__(256) k_ucells(Grid2 G, const double4 *__restrict__ cur,
                                                const double4 *__restrict__ un, double4 *next,
                                                const double4 *__restrict__ Fx, const double4 *__restrict__ Fy,
                                                double g, double cxa, double cxb, double cya, double cyb,
                                                double tstep, int krk) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)G.nx * G.ny) return;
    const int r = (int)(t / G.nx), i = (int)(t % G.nx);
    const int row = 3 + r, col = 3 + i;
    const int64_t self = G.at(row, col);
    const Prim q = load_prim(cur, self);
    const Prim qp = load_prim(cur, G.at(row, col + 1)), qm = load_prim(cur, G.at(row, col - 1));
    const Prim rp = load_prim(cur, G.at(row + 1, col)), rmn = load_prim(cur, G.at(row - 1, col));
    const double4 fxr = Fx[(int64_t)r * (G.nx + 1) + i + 1], fxl = Fx[(int64_t)r * (G.nx + 1) + i];
    const double4 fyr = Fy[(int64_t)(r + 1) * G.nx + i], fyl = Fy[(int64_t)r * G.nx + i];
    double Ep[4], Em[4], Gp[4], Gm[4];
    phys_flux<0>(qp, g, Ep);
    phys_flux<0>(qm, g, Em);
    phys_flux<1>(rp, g, Gp);
    phys_flux<1>(rmn, g, Gm);
    const double FR[4] = {fxr.x, fxr.y, fxr.z, fxr.w}, FL[4] = {fxl.x, fxl.y, fxl.z, fxl.w};
    const double HR[4] = {fyr.x, fyr.y, fyr.z, fyr.w}, HL[4] = {fyl.x, fyl.y, fyl.z, fyl.w};
    double U[4];
    U[0] = q.r;
    U[1] = q.r * q.u;
    U[2] = q.r * q.v;
    U[3] = q.p / (g - 1.0) + 0.5 * q.r * (q.u * q.u + q.v * q.v);
    double Ut[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const double dE = cxa * (FR[n] - FL[n]) - cxb * (Ep[n] - Em[n]);
        const double dF = cya * (HR[n] - HL[n]) - cyb * (Gp[n] - Gm[n]);
        const double fu = -dE - dF;
        Ut[n] = U[n] + fu * tstep;
    }
    const double r0 = Ut[0];
    const double u0 = Ut[1] / Ut[0];
    const double v0 = Ut[2] / Ut[0];
    const double p0 = (g - 1.0) * r0 * (Ut[3] / r0 - 0.5 * (u0 * u0 + v0 * v0));
    const double4 n0 = un[self];
    const double ra = krk == 1 ? 0.0 : krk == 2 ? 3.0 / 4.0 : 1.0 / 3.0;
    const double rb = krk == 1 ? 1.0 : krk == 2 ? 1.0 / 4.0 : 2.0 / 3.0;
    next[self] = make_double4(ra * n0.x + rb * r0, ra * n0.y + rb * u0, ra * n0.z + rb * v0, ra * n0.w + rb * p0);
}

// periodic ghost fill (BC_cyc at level 0, src/solution.F90:116-136);
// corners are left alone, as the reference never refills them
__global__ void k_ughosts(Grid2 G, double4 *buf) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int H = G.ny + 6;
    if (t >= (int64_t)G.W * H) return;
    const int row = (int)(t / G.W), col = (int)(t % G.W);
    const bool gx = col < 3 || col > G.nx + 2, gy = row < 3 || row > G.ny + 2;
    if (gx == gy) return;   // interior or corner
    int sr = row, sc = col;
    if (col < 3) sc = col + G.nx;
    else if (col > G.nx + 2) sc = col - G.nx;
    if (row < 3) sr = row + G.ny;
    else if (row > G.ny + 2) sr = row - G.ny;
    buf[t] = buf[G.at(sr, sc)];
}

__global__ void k_ucorners(Grid2 G, const double4 *__restrict__ in, double4 *out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int H = G.ny + 6;
    if (t >= (int64_t)G.W * H) return;
    const int row = (int)(t / G.W), col = (int)(t % G.W);
    const bool gx = col < 3 || col > G.nx + 2, gy = row < 3 || row > G.ny + 2;
    if (gx && gy) out[t] = in[t];
}

static inline unsigned nb(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace uniform_static
}  // namespace fdm

extern "C" int fdm_time_advance_rk_uniform_static(const double *prim_in, double *prim_out, int32_t nx,
                                                  int32_t ny, double h, double x_factor, double gama,
                                                  double lambda_x, double lambda_y, double tstep,
                                                  void *stream) {
    using namespace fdm::uniform_static;
    if (!prim_in || !prim_out) return FDM_ERR_ARG;
    if (nx < 3 || ny < 3 || nx > FDM_STATIC_MAX_SIDE || ny > FDM_STATIC_MAX_SIDE ||
        (int64_t)nx * ny > FDM_STATIC_MAX_CELLS)
        return FDM_ERR_ARG;   // outside the fixed scratch: nothing was enqueued
    const int64_t ngrid = (int64_t)(nx + 6) * (ny + 6);
    const int64_t nface = std::max((int64_t)(nx + 1) * ny, (int64_t)nx * (ny + 1));
    if (ngrid > GRID_CAP || nface > FACE_CAP) return FDM_ERR_ARG;
    if (((uintptr_t)prim_in | (uintptr_t)prim_out) & 31) return FDM_ERR_ARG;   // 32-byte records
    // stage 3 reads prim_in while it writes prim_out, and the corners are
    // copied from prim_in last: the two ranges must not share a byte
    const uintptr_t ia = (uintptr_t)prim_in, oa = (uintptr_t)prim_out, nbytes = (uintptr_t)ngrid * 32;
    if (ia < oa + nbytes && oa < ia + nbytes) return FDM_ERR_ARG;
    // an error left pending by earlier, unrelated work is the caller's, not
    // this call's: refuse before enqueueing anything rather than report it
    if (cudaPeekAtLastError() != cudaSuccess) return FDM_ERR_CUDA;
    double4 *base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return FDM_ERR_CUDA;
    double4 *U1 = base, *U2 = base + GRID_CAP, *Fx = base + 2 * GRID_CAP, *Fy = Fx + FACE_CAP;
    cudaStream_t s = (cudaStream_t)stream;
    Grid2 G{nx, ny, nx + 6};
    const double dy = h, dx = x_factor * dy;
    const double cxa = 4.0 / (3.0 * dx), cxb = 1.0 / (6.0 * dx);
    const double cya = 4.0 / 3.0 / dy, cyb = 1.0 / 6.0 / dy;
    const double4 *in = (const double4 *)prim_in;
    double4 *out = (double4 *)prim_out;
    const double4 *cur[3] = {in, U1, U2};
    double4 *next[3] = {U1, U2, out};
    for (int krk = 1; krk <= 3; ++krk) {
        k_ufaces<0><<<nb((int64_t)(nx + 1) * ny, 128), 128, 0, s>>>(G, cur[krk - 1], Fx, gama, lambda_x);
        k_ufaces<1><<<nb((int64_t)nx * (ny + 1), 128), 128, 0, s>>>(G, cur[krk - 1], Fy, gama, lambda_y);
        k_ucells<<<nb((int64_t)nx * ny, 256), 256, 0, s>>>(G, cur[krk - 1], in, next[krk - 1], Fx, Fy, gama, cxa,
                                                           cxb, cya, cyb, tstep, krk);
        k_ughosts<<<nb(ngrid, 256), 256, 0, s>>>(G, next[krk - 1]);
    }
    k_ucorners<<<nb(ngrid, 256), 256, 0, s>>>(G, in, out);
    return cudaGetLastError() == cudaSuccess ? FDM_OK : FDM_ERR_CUDA;
}
