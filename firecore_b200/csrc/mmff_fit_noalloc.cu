// mmff_fit_noalloc.cu -- in-place cubic B-spline fit of a caller-owned device
// grid that allocates nothing.
//
// Who needs it: code that may not allocate device memory at the point where
// it wants a fit -- a runtime that hands out all device memory from its own
// fixed arena (and treats any cudaMalloc as an error because it would
// fragment or oversubscribe the arena), or a host thread that runs while
// another part of the program holds the device allocator.  mmff_grid_build
// allocates its potential and work buffers with cudaMalloc; this entry point
// works on the caller's array only.
//
// The three 1-D solves of the fit (periodic along x and y, zero coefficients
// outside the grid along z) share per-axis elimination coefficients that
// depend only on the axis length.  They are computed once per call into
// g_fit_scratch, a file-scope device array that every GPU loading this
// library holds until the process exits, then every grid line is solved with
// them.  Limit: each axis at most MMFF_FIT_NMAX points.
#include <cuda_runtime.h>
#include <cstdio>
#include <string>

#include "mmff_host.h"

#define MMFF_FIT_NMAX 4096

// per axis: cp[NMAX], z[NMAX], then scalars (zden) -- 3 axes
static __device__ __align__(256) double g_fit_scratch[3 * 3 * MMFF_FIT_NMAX];

namespace {

// cp (and for periodic axes z, zden) of the solve of (c[i-1] + 4c[i] + c[i+1])/6 = v[i]
__global__ void fit_coef_kernel(double* scr, int nx, int ny, int nz) {
    const int axis = threadIdx.x;           // 0: z (open), 1: y, 2: x (periodic)
    if (axis > 2) return;
    const int n = axis == 0 ? nz : (axis == 1 ? ny : nx);
    double* cp = scr + axis * 3 * MMFF_FIT_NMAX;
    double* z = cp + MMFF_FIT_NMAX;
    double* sc = cp + 2 * MMFF_FIT_NMAX;
    const double a = 1.0 / 6.0, b = 4.0 / 6.0;
    if (axis == 0) {
        cp[0] = a / b;
        for (int i = 1; i < n; i++) cp[i] = a / (b - a * cp[i - 1]);
        return;
    }
    const double gamma = -b, bb0 = b - gamma, bbn = b - a * a / gamma;
    cp[0] = a / bb0;
    z[0] = gamma / bb0;
    for (int i = 1; i < n; i++) {
        const double diag = (i == n - 1 ? bbn : b) - a * cp[i - 1];
        cp[i] = a / diag;
        const double ui = (i == n - 1) ? a : 0.0;
        z[i] = (ui - a * z[i - 1]) / diag;
    }
    for (int i = n - 2; i >= 0; i--) z[i] -= cp[i] * z[i + 1];
    sc[0] = 1.0 + z[0] + a * z[n - 1] / gamma;
}

__global__ void fit_open_kernel(double* __restrict__ C, long nlines, int n, long line_stride, long elem_stride,
                                int nlines_inner, long inner_stride, const double* __restrict__ scr) {
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const double* cp = scr;
    const long base = (l / nlines_inner) * line_stride + (l % nlines_inner) * inner_stride;
    const double a = 1.0 / 6.0, b = 4.0 / 6.0;
    for (int ch = 0; ch < 3; ch++) {
        double* y = C + ch;
        y[3 * base] = y[3 * base] / b;
        for (int i = 1; i < n; i++) {
            const double diag = b - a * cp[i - 1];
            const long k = base + i * elem_stride, km = base + (i - 1) * elem_stride;
            y[3 * k] = (y[3 * k] - a * y[3 * km]) / diag;
        }
        for (int i = n - 2; i >= 0; i--) {
            const long k = base + i * elem_stride, kp = base + (i + 1) * elem_stride;
            y[3 * k] -= cp[i] * y[3 * kp];
        }
    }
}

__global__ void fit_periodic_kernel(double* __restrict__ C, long nlines, int n, long line_stride, long elem_stride,
                                    int nlines_inner, long inner_stride, const double* __restrict__ scr) {
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const double* cp = scr;
    const double* z = scr + MMFF_FIT_NMAX;
    const double zden = scr[2 * MMFF_FIT_NMAX];
    const long base = (l / nlines_inner) * line_stride + (l % nlines_inner) * inner_stride;
    const double a = 1.0 / 6.0, b = 4.0 / 6.0;
    const double gamma = -b, bb0 = b - gamma, bbn = b - a * a / gamma;
    for (int ch = 0; ch < 3; ch++) {
        double* y = C + ch;
        y[3 * base] = y[3 * base] / bb0;
        for (int i = 1; i < n; i++) {
            const double diag = (i == n - 1 ? bbn : b) - a * cp[i - 1];
            const long k = base + i * elem_stride, km = base + (i - 1) * elem_stride;
            y[3 * k] = (y[3 * k] - a * y[3 * km]) / diag;
        }
        for (int i = n - 2; i >= 0; i--) {
            const long k = base + i * elem_stride, kp = base + (i + 1) * elem_stride;
            y[3 * k] -= cp[i] * y[3 * kp];
        }
        const long klast = base + (long)(n - 1) * elem_stride;
        const double fact = (y[3 * base] + a * y[3 * klast] / gamma) / zden;
        for (int i = 0; i < n; i++) y[3 * (base + i * elem_stride)] -= fact * z[i];
    }
}

int fit_fail(const char* msg, cudaError_t e = cudaSuccess) {
    std::string m = msg;
    if (e != cudaSuccess) { m += ": "; m += cudaGetErrorString(e); }
    mmff_set_error(m.c_str());   // reported by mmff_last_error()
    return -1;
}

}  // namespace

extern "C" {

// In-place fit of coefs [nx][ny][nz][3] (device memory, FP64, z fastest): on
// entry the node values, on exit the B-spline coefficients.  See the file
// comment for who calls this and why; limits and the shared scratch are
// documented in include/MMFFmulti_lib.h.
int mmff_bspline_fit_noalloc(double* d_coefs, int nx, int ny, int nz, void* stream) {
    if (!d_coefs) return fit_fail("mmff_bspline_fit_noalloc: null grid pointer");
    if (nx < 3 || ny < 3 || nz < 2) return fit_fail("mmff_bspline_fit_noalloc: grid too small (need nx, ny >= 3, nz >= 2)");
    if (nx > MMFF_FIT_NMAX || ny > MMFF_FIT_NMAX || nz > MMFF_FIT_NMAX) {
        char buf[160];
        snprintf(buf, sizeof buf, "mmff_bspline_fit_noalloc: grid %dx%dx%d exceeds the %d points per axis this entry point supports",
                 nx, ny, nz, MMFF_FIT_NMAX);
        return fit_fail(buf);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fit_fail("mmff_bspline_fit_noalloc: cudaGetDevice", e);
    // the grid must be device (or managed) memory of the current device: a
    // host pointer or another GPU's buffer is an argument error here, not a
    // fault inside the solve kernels (the query allocates nothing)
    cudaPointerAttributes pa;
    e = cudaPointerGetAttributes(&pa, d_coefs);
    if (e != cudaSuccess) { cudaGetLastError(); return fit_fail("mmff_bspline_fit_noalloc: grid pointer not known to CUDA", e); }
    if ((pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) || pa.device != dev)
        return fit_fail("mmff_bspline_fit_noalloc: grid pointer is not device memory of the current device");
    // device address of the scratch array on the current device, taken on
    // every call (it allocates nothing): the host-side name g_fit_scratch is
    // only a stand-in, and an address kept from an earlier call would be
    // stale after the program reset or recreated this device's context
    double* scr = nullptr;
    e = cudaGetSymbolAddress((void**)&scr, g_fit_scratch);
    if (e != cudaSuccess || !scr) return fit_fail("mmff_bspline_fit_noalloc: cudaGetSymbolAddress", e);
    cudaStream_t st = (cudaStream_t)stream;
    fit_coef_kernel<<<1, 32, 0, st>>>(scr, nx, ny, nz);
    const long lz = (long)nx * ny, ly = (long)nx * nz, lx = (long)ny * nz;
    fit_open_kernel<<<(unsigned)((lz + 127) / 128), 128, 0, st>>>(d_coefs, lz, nz, nz, 1, 1, 0, scr);
    fit_periodic_kernel<<<(unsigned)((ly + 127) / 128), 128, 0, st>>>(d_coefs, ly, ny, (long)ny * nz, nz, nz, 1,
                                                                      scr + 3 * MMFF_FIT_NMAX);
    fit_periodic_kernel<<<(unsigned)((lx + 127) / 128), 128, 0, st>>>(d_coefs, lx, nx, 1, (long)ny * nz, 1, 0,
                                                                      scr + 6 * MMFF_FIT_NMAX);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fit_fail("mmff_bspline_fit_noalloc: launch", e);
    return 0;
}

}  // extern "C"
