// Kernels of the differentiable model: the weighted Poisson negative
// log-likelihood of the UPDC forward model and the pieces of its gradient.
//
//   mu_k = S_k P_k x + (background_k + pedestal_k),  y_k = SCI_k + pedestal_k
//   L    = sum_k sum_p W_kp (mu_kp - y_kp log mu_kp)
//   dL/dmu_kp = W_kp (1 - y_kp / mu_kp) =: r_kp
// so dL/dx = sum_k H_k^T r_k (the engine's adjoint path applied to r),
// dL/dbackground_k = sum_p r_kp, dL/dpedestal_k = sum_p (r_kp - W_kp log mu_kp),
// and dL/dpsi_k[j] = sum_t (S_k^T r_k)[t] x[t - j + c] for the normalised PSF.
// A pixel enters only where W > 0 and mu > 0 (the log is undefined
// elsewhere; such pixels are counted and get r = 0, as FreezeMu gives them
// ratio 1 in the solver, updc_core.c:1163-1166).
#pragma once

#include "pointwise.cuh"

namespace updc {

constexpr int NLL_TERMS = 4;  // sum W(mu - y log mu), sum r, sum W log mu, pixels with W > 0 and mu <= 0

// One exposure per blockIdx.y; per-block FP64 partial sums in
// part[(k * gridDim.x + block) * NLL_TERMS + i], reduced on the host in
// block order (deterministic).
template <typename T>
__global__ void __launch_bounds__(256) k_nll(const ExpDesc<T> *__restrict__ exps, size_t nin, size_t nout,
                                             const T *__restrict__ blur_all, T *__restrict__ r_all,
                                             double *__restrict__ part) {
    const int k = blockIdx.y;
    const ExpDesc<T> e = exps[k];
    const T *blur = blur_all + (size_t)k * nout;
    T *r = r_all + (size_t)k * nin;
    double acc[NLL_TERMS] = {0, 0, 0, 0};
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < nin; p += (size_t)gridDim.x * blockDim.x) {
        const double w = (double)e.wht[p];
        double rv = 0;
        if (w > 0) {
            double pred = 0;
            const uint32_t z0 = e.off[p], z1 = e.off[p + 1];
            for (uint32_t z = z0; z < z1; ++z) {
                const uint32_t t = e.delta16 ? e.base[p] + e.delta[z] : e.tgt[z];
                pred = __fma_rn((double)e.frac[z], (double)blur[t < nout ? t : 0], pred);
            }
            const double mu = pred + ((double)e.background + (double)e.pedestal);
            const double y = (double)e.sci[p] + (double)e.pedestal;
            if (mu > 0) {
                const double lg = log(mu);
                rv = w * (1.0 - y / mu);
                acc[0] += w * (mu - y * lg);
                acc[1] += rv;
                acc[2] += w * lg;
            } else {
                acc[3] += 1.0;
            }
        }
        r[p] = (T)rv;
    }
    __shared__ double s[NLL_TERMS][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < NLL_TERMS; ++i) {
        const double v = block_sum_warp(acc[i]);
        if (lane == 0) s[i][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NLL_TERMS) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[threadIdx.x][w];
        part[((size_t)k * gridDim.x + blockIdx.x) * NLL_TERMS + threadIdx.x] = t;
    }
}

// a[i] *= conj(b[i])  (cross-correlation spectrum)
template <typename T>
__global__ void k_mul_conj(cx<T> *__restrict__ a, const cx<T> *__restrict__ b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const cx<T> u = a[i], v = b[i];
        a[i] = {u.x * v.x + u.y * v.y, u.y * v.x - u.x * v.y};
    }
}

// Row C2R epilogue that keeps only the lags of a PSF window: output (y, x)
// is the lag m = (y, x) of the circular correlation, PSF pixel
// ((y + fhei/2) mod FH, (x + fwid/2) mod FW), the inverse of PsfLoader's
// centre wrap (updc_core.c:826-833).
template <typename T> struct PsfWindowStore {
    double *out;
    int pw, fwid, fhei, FW, FH, transposed;
    __device__ __forceinline__ void operator()(int, int yy, int xx, T v) const {
        const int y = (yy + fhei / 2) % FH, x = (xx + fwid / 2) % FW;
        if (y >= fhei || x >= fwid) return;
        const size_t dst = transposed ? (size_t)x * pw + y : (size_t)y * pw + x;
        out[dst] = (double)v;
    }
};

}  // namespace updc
